"""The oracle's proposed-interval semantics (CPU): an interval that starts at
or before a ray's first hit, or holds no hit, leaves the march unchanged; a
t_near beyond the first hits removes exactly those hits."""
import numpy as np

from scenes_for_tests import dense_scene, dense_view

H, W = 24, 32


def test_interval_semantics(oracle):
    sc = dense_scene(seed=2, P=1500)
    ro, rd = dense_view(H=H, W=W)
    plain = oracle.forward(sc, ro, rd, nthreads=8)
    ids, ts, cnt = oracle.hit_stream(sc, ro, rd, max_hits=64, nthreads=8)
    hit = (cnt > 0).reshape(H, W)
    assert hit.mean() > 0.5
    first = np.where(cnt > 0, ts[:, 0], 0.0).reshape(H, W).astype(np.float32)
    for iv in (np.stack([first, np.full((H, W), np.inf, np.float32)]),      # starts at the first hit
               np.stack([first, first]),                                    # t_far does not matter
               np.full((2, H, W), [[[500.0]], [[600.0]]], np.float32),      # no hit inside: plain
               np.full((2, H, W), np.nan, np.float32)):                     # ignored
        got = oracle.forward(sc, ro, rd, nthreads=8, interval=iv)
        np.testing.assert_array_equal(got.color, plain.color)
        np.testing.assert_array_equal(got.others, plain.others)
    # t_near just past the first hit: that hit (and any tie before it) is skipped
    nxt = np.nextafter(first, np.float32(np.inf))
    iv = np.stack([np.where(hit, nxt, 0.0), np.full((H, W), np.inf)]).astype(np.float32)
    got = oracle.forward(sc, ro, rd, nthreads=8, interval=iv)
    changed = np.abs(got.color - plain.color).max(axis=0) > 0
    assert changed[hit].mean() > 0.5 and not changed[~hit].any()
    # ... and equals the march of the hits from the second one on, starting a fresh chunk there
    b = oracle.backward(sc, ro, rd, got.color, got.others, np.ones((3, H, W), np.float32),
                        np.zeros((7, H, W), np.float32), nthreads=8, interval=iv)
    assert np.isfinite(b.dsh).all() and np.abs(b.dsh).sum() > 0
