"""Compares the k-closest queries the reference's own code made (its any-hit
program's 16-slot payload after each optixTrace, logged by the host build of
tritracer/closestk.h:17-149 through oracle/refshim) with a hit stream: every
hit of the ray in [0, 1000] ordered by (t, primitive id).

For each logged query with lower bound tmin, the payload must hold the first
16 hits of the stream at t >= tmin (closed interval) or t > tmin (open), with
the same t values in the same order; within a group of hits at one exact t
the order is the reference's traversal order, so only the sets must agree,
and a group cut off by the 16th slot may keep any of its members.
"""
from __future__ import annotations

import numpy as np

INVALID = 0xFFFFFFFF


def compare_chunks(chunk_ids, chunk_tmin, chunk_count, ids, ts, counts, closed: bool, max_hits: int):
    """Returns (queries compared, queries whose order differed only inside
    groups of equal t). Raises AssertionError on any other difference."""
    R, C, _ = chunk_ids.shape
    compared = tie_reordered = 0
    for r in range(R):
        n_stream = int(counts[r])
        if n_stream > max_hits:  # the stream holds only the first max_hits hits
            n_stream = max_hits
            complete = False
        else:
            complete = True
        s_ids = ids[r, :n_stream].astype(np.uint32)
        s_t = ts[r, :n_stream].astype(np.float32)
        t_of = {int(i): t for i, t in zip(s_ids, s_t)}
        for c in range(min(int(chunk_count[r]), C)):
            tmin = np.float32(chunk_tmin[r, c])
            start = int(np.searchsorted(s_t, tmin, side="left" if closed else "right"))
            want_ids = s_ids[start:start + 16]
            if not complete and start + 16 > n_stream:
                continue  # the stream does not reach this query's window
            got = chunk_ids[r, c]
            got = got[got != INVALID]
            assert len(got) == len(want_ids), (r, c, len(got), len(want_ids))
            if len(got) == 0:
                compared += 1
                continue
            assert all(int(i) in t_of for i in got), (r, c, "a reference hit missing from the stream")
            got_t = np.array([t_of[int(i)] for i in got], np.float32)
            want_t = s_t[start:start + len(got)]
            np.testing.assert_array_equal(got_t.view(np.uint32), want_t.view(np.uint32), err_msg=f"ray {r} query {c}")
            last_t = want_t[-1]
            full = len(got) == 16
            for t in np.unique(want_t):
                g = set(int(i) for i, tt in zip(got, got_t) if tt == t)
                if full and t == last_t:
                    pool = set(int(i) for i, tt in zip(s_ids, s_t) if tt == t)
                    assert g <= pool, (r, c, "cut-off tie group")
                else:
                    w = set(int(i) for i, tt in zip(want_ids, want_t) if tt == t)
                    assert g == w, (r, c, float(t))
            if not np.array_equal(got, want_ids):
                tie_reordered += 1
            compared += 1
    return compared, tie_reordered
