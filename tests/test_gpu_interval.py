"""Proposed intervals and hit records through the C ABI (tt_view.interval /
tt_view.record), the traversal clipping that the proposal network drives.

* The record of a plain forward holds each ray's first and last visited hit
  and whether it terminated.
* Intervals that hold every hit the plain march visits (the recorded ones, a
  t_far that is too short, an interval without hits, NaN) give the plain
  results BIT FOR BIT: a ray that reaches t_far unterminated continues beyond
  it, a ray without a hit in its interval is traced again without it.
* An interval whose t_near skips hits gives what the FP64 oracle gives for
  the same interval (same tolerances as the plain parity tests).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, scenes  # noqa: E402
from gpu_helpers import DEV, MARGIN, T, flagged_prims, rel_norm  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL = 1e-5, 1e-6
GRAD_RTOL = 1e-4
H, W = 48, 64


def scene_tensors(sc):
    return dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
                shs=T(sc.shs), opac=T(sc.opacities))


def run(tr, sc, s, ro, rd, g, go, interval=None, record=False):
    """Forward (+ record) and adjoint of one view with the same interval."""
    bg = torch.zeros(3, device=DEV)
    scaling = torch.zeros(sc.P, device=DEV)
    density = torch.zeros(sc.P, device=DEV)
    rec = torch.empty((3, H, W), device=DEV) if record else None
    iv = None if interval is None else [T(np.ascontiguousarray(interval, np.float32))]
    outs, maxb = tr.trace_forward_views([(T(ro), T(rd))], s["verts"], s["sigma"], s["npts"], s["cums"], sc.P,
                                        s["shs"], 3, s["opac"], scaling, density, bg, 0, intervals=iv,
                                        records=None if rec is None else [rec])
    grads = tr.trace_backward_views([(T(ro), T(rd))], outs, [(T(g), T(go))], s["verts"], s["sigma"], s["npts"],
                                    s["cums"], sc.P, s["shs"], 3, s["opac"], bg, intervals=iv)
    torch.cuda.synchronize()
    tr.device_status()
    col, oth = outs[0]
    out = dict(color=col.cpu().numpy(), others=oth.cpu().numpy(), max_blending=maxb.cpu().numpy(),
               density=density.cpu().numpy(), scaling=scaling.cpu().numpy(),
               grads=[x.cpu().numpy() for x in grads])
    if rec is not None:
        out["record"] = rec.cpu().numpy()
    return out


@pytest.fixture(scope="module")
def setup():
    sc = dense_scene(seed=2, P=3000)
    ro, rd = dense_view(H=H, W=W)
    g, go = scenes.upstream_grads(H, W, seed=3, others_std=1.0)
    return sc, scene_tensors(sc), ro, rd, g, go


def assert_same(a, b):
    for key in ("color", "others", "max_blending", "density", "scaling"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    for x, y in zip(a["grads"], b["grads"]):
        assert rel_norm(x, y) < 1e-6  # float atomics: only the summation order differs


@pytest.mark.parametrize("traversal", ["packets", "lanes"])
def test_record_then_intervals_reproduce_plain(setup, traversal):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal)
    plain = run(tr, sc, s, ro, rd, g, go, record=True)
    rec = plain["record"]
    hit = np.isfinite(rec[0])
    assert hit.mean() > 0.5
    # the record: first hit of the plain hit stream, ordered, alpha channel of terminated rays
    _, ts, cnt = [x.cpu().numpy() for x in tr.hit_stream(T(ro), T(rd), max_hits=4)]
    first = np.where(cnt > 0, ts[:, 0], np.inf).reshape(H, W)
    np.testing.assert_array_equal(rec[0], first)  # no hit before the near plane in this view
    assert np.all(rec[1][hit] >= rec[0][hit])
    term = rec[2] == 1.0
    assert term.sum() > 50 and (~term & hit).sum() > 50
    assert np.all(plain["others"][1][term] > 0.99)  # T < 1e-4 / (1 - 0.99)

    cases = {
        "recorded": rec[:2],
        "short_far": np.stack([rec[0], rec[0]]),               # every hit after the first comes by continuation
        "no_hit": np.full((2, H, W), [[[500.0]], [[600.0]]]),  # nothing inside: traced again
        "nan": np.full((2, H, W), np.nan),                     # ignored
        "inverted": np.stack([rec[1], rec[0] * 0.5]),          # t_far < t_near: traced again
    }
    for name, iv in cases.items():
        tr.reset_stats()
        got = run(tr, sc, s, ro, rd, g, go, interval=iv)
        st = tr.stats()
        assert_same(got, plain)
        n_hit, n_open = int(hit.sum()), int((hit & ~term).sum())
        if name == "recorded":
            assert st["interval_continuations"] == n_open and st["interval_retraces"] == 0, (name, st)
        if name == "no_hit":
            assert st["interval_retraces"] == H * W and st["interval_continuations"] == 0, (name, st)
        if name == "inverted":
            assert st["interval_retraces"] == n_hit, (name, st)


def test_late_near_matches_oracle(oracle, setup):
    """t_near between the first and last hit: the skipped hits are absent in
    the GPU result exactly as in the FP64 oracle given the same interval."""
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    plain = run(tr, sc, s, ro, rd, g, go, record=True)
    rec = plain["record"]
    hit = np.isfinite(rec[0])
    iv = np.stack([np.where(hit, 0.5 * (rec[0] + rec[1]), 0.0), np.full((H, W), np.inf)]).astype(np.float32)
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=256, nthreads=8, interval=iv)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.mean() > 0.97
    gm, gom = g * ok[None], go * ok[None]
    got = run(tr, sc, s, ro, rd, gm, gom, interval=iv)
    changed = np.abs(got["color"] - plain["color"]).max(axis=0) > 1e-3
    assert changed.sum() > 100  # the clip really removed hits
    for key in ("color", "others"):
        a, b = got[key][:, ok], getattr(ref, key)[:, ok]
        assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL), key
    skip = np.zeros(sc.P, bool)
    skip[flagged_prims(ref, H, W, ok)] = True
    np.testing.assert_array_equal(got["density"][~skip], ref.density[~skip])
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, gm, gom, precision=64, exact=True, canonical=True,
                         nthreads=8, interval=iv)
    for key, x in zip(("dtri", "dsigma", "dopac", "dsh"), got["grads"]):
        e = rel_norm(x, getattr(rb, key))
        assert e < GRAD_RTOL, (key, e)


def test_interval_shape_checked(setup):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    with pytest.raises(ValueError, match="interval"):
        run(tr, sc, s, ro, rd, g, go, interval=np.zeros((2, H, W + 1), np.float32))
