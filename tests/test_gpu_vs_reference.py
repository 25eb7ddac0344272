"""The CUDA path against the reference's own code, on the same inputs.

The reference's device programs (tritracer/forward.cu, backward.cu,
closestk.h) compiled for the host from their files (oracle/_ref, built by
oracle/Makefile), with the restated watertight intersector and CPU BVH
standing in for OptiX's closed traversal, are run on the same scenes and
rays as the GPU:

* queries: every k-closest query the reference's any-hit program answered
  (its 16-slot payload, logged per ray) holds the same hits, in the same t
  order, as the GPU's hit stream from that query's lower bound on: the
  hit-index sequences are identical except for the order inside groups of
  hits at exactly the same t;
* numbers, in two shading modes of the GPU:
  - reference arithmetic (tt_config.reference_arithmetic = 1: the hit point
    o + t d and the window function in FP32 as the reference evaluates them):
    images within 1e-5 relative (|d| <= 1e-5 |ref| + 1e-6 per pixel) and
    gradients within 1e-4 relative (L2) of the reference's;
  - the default mode (hit point from an FP64 ray/plane solve): its error
    against the reference's code is measured and printed beside its error
    against the FP64 oracle. It is bounded loosely here: the reference's FP32
    edge distances on small triangles far from the origin keep only ~3
    digits, so the reference itself is that far from the FP64 answer.
`scaling` is written by the first ray that blends a triangle (a race in the
reference too); it is compared for the one-camera cases, where every such
ray starts at the same origin. Rays whose FP32 threshold decisions (alpha
vs 1/255, T(1 - alpha) vs 1e-4) lie within 1e-5 (relative) of flipping are
left out of the per-pixel checks,
and their upstream gradients are zero.

Cases: the dense 3k-triangle scene, the random 20k-triangle scene, and a
seeded sample of 4096 pixels of the 1M-triangle, 4 x 800 x 800 benchmark
workload (rays are independent, so the sample is traced as an image of its
own over the full scene).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, scenes  # noqa: E402
from gpu_helpers import MARGIN, T, flagged_prims, gpu_backward, gpu_forward, rel_norm, settings  # noqa: E402
from ref_chunks import compare_chunks  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL, GRAD_RTOL = 1e-5, 1e-6, 1e-4
BG = np.array([0.1, 0.2, 0.3], np.float32)
MAX_HITS = 256


def c2_sample(n=4096, seed=7):
    sc = scenes.make_scene(1_000_000, seed=0)
    rays = [scenes.camera_rays(c) for c in scenes.sphere_cameras(4, 800, 800, seed=0)]
    ro = np.concatenate([r[0].reshape(-1, 3) for r in rays], 0)
    rd = np.concatenate([r[1].reshape(-1, 3) for r in rays], 0)
    idx = np.sort(np.random.default_rng(seed).choice(ro.shape[0], n, replace=False))
    side = int(np.sqrt(n))
    return sc, (ro[idx].reshape(side, n // side, 3).copy(), rd[idx].reshape(side, n // side, 3).copy())


def cases():
    yield "dense3k", dense_scene(seed=1, P=3000), dense_view(H=48, W=64)
    sc = scenes.make_scene(20000, seed=5)
    yield "random20k", sc, scenes.camera_rays(scenes.sphere_cameras(1, 56, 72, seed=5)[0])


CASES = list(cases())


@pytest.fixture(scope="module")
def c2():
    return c2_sample()


def all_cases(c2):
    return CASES + [("c2_sample", c2[0], c2[1])]


def hit_stream(sc, ro, rd):
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.build_tri_accel(T(sc.verts), T(sc.cumsum), sc.P, True)
    ids, ts, cnt = [x.cpu().numpy() for x in tr.hit_stream(T(ro), T(rd), max_hits=MAX_HITS)]
    tr.device_status()
    return ids, ts, cnt


@pytest.mark.parametrize("incl", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("which", ["dense3k", "random20k", "c2_sample"])
def test_queries_equal_the_references(reference, c2, which, incl):
    if which == "c2_sample" and not incl:
        pytest.skip("one convention is enough at full scale")
    name, sc, (ro, rd) = next(c for c in all_cases(c2) if c[0] == which)
    f = reference.forward(sc, ro, rd, bg=BG, tmin_inclusive=incl, chunks=12, nthreads=8)
    ids, ts, cnt = hit_stream(sc, ro, rd)
    n, reordered = compare_chunks(f.chunk_ids, f.chunk_tmin, f.chunk_count, ids, ts, cnt, incl, MAX_HITS)
    print(f"{name} ({'closed' if incl else 'open'}): {n} reference queries equal the GPU hit stream; "
          f"{reordered} differ only by the order of hits at equal t")
    assert n >= ro.shape[0] * ro.shape[1]  # at least one query per ray was compared


def decisions_ok(oracle, sc, ro, rd, incl=True):
    """Rays whose FP32 threshold decisions are clear of flipping (the FP32
    oracle is bit-identical to the reference's code)."""
    H, W = ro.shape[:2]
    r = oracle.forward(sc, ro, rd, bg=BG, precision=32, tmin_inclusive=incl, record=256, nthreads=8)
    return (r.margin > MARGIN).reshape(H, W), r


def image_err(got, want, ok):
    a, b = got[:, ok], want[:, ok]
    err = np.abs(a - b)
    return float(err.max()), float((err / (RTOL * np.abs(b) + ATOL)).max()), float(np.sqrt((err ** 2).mean()))


@pytest.mark.parametrize("which", ["dense3k", "random20k", "c2_sample"])
def test_forward_vs_reference(oracle, reference, c2, which):
    name, sc, (ro, rd) = next(c for c in all_cases(c2) if c[0] == which)
    H, W = ro.shape[:2]
    ok, rec = decisions_ok(oracle, sc, ro, rd)
    assert ok.mean() > 0.97, ok.mean()
    ref = reference.forward(sc, ro, rd, bg=BG, nthreads=8)
    f64 = oracle.forward(sc, ro, rd, bg=BG, precision=64, exact=True, canonical=True, nthreads=8)
    st = settings(bg=BG)
    for mode in ("reference_arithmetic", "default"):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", reference_arithmetic=(mode != "default"))
        out = gpu_forward(tr, sc, ro, rd, st)
        tr.device_status()
        for key in ("color", "others"):
            mx, worst, rms = image_err(out[key], getattr(ref, key), ok)
            mx64, worst64, rms64 = image_err(out[key], getattr(f64, key), ok)
            print(f"{name} {mode} {key}: vs the reference's code max |d| {mx:.2e} (worst/tol {worst:.3g}, "
                  f"rms {rms:.2e}); vs the FP64 oracle max |d| {mx64:.2e} (worst/tol {worst64:.3g}, rms {rms64:.2e})")
            if mode == "reference_arithmetic":
                assert worst <= 1.0, (key, worst)
            else:
                assert mx < 2e-2 and rms < 1e-3, (key, mx, rms)
        if mode == "reference_arithmetic":
            skip = np.zeros(sc.P, bool)
            skip[flagged_prims(rec, H, W, ok)] = True
            np.testing.assert_array_equal(out["density"][~skip], ref.density[~skip])
            np.testing.assert_allclose(out["max_blending"][~skip], ref.max_blending[~skip], rtol=RTOL, atol=ATOL)
            if name != "c2_sample":  # one camera: every ray that may write a triangle's scaling agrees
                np.testing.assert_allclose(out["scaling"][~skip], ref.scaling[~skip], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("which", ["dense3k", "random20k", "c2_sample"])
def test_backward_vs_reference(oracle, reference, c2, which):
    name, sc, (ro, rd) = next(c for c in all_cases(c2) if c[0] == which)
    H, W = ro.shape[:2]
    ok, _ = decisions_ok(oracle, sc, ro, rd)
    g, go = scenes.upstream_grads(H, W, seed=11, others_std=1.0)
    g = np.ascontiguousarray(g * ok[None])
    go = np.ascontiguousarray(go * ok[None])
    st = settings()
    f = reference.forward(sc, ro, rd, nthreads=8)
    ref = reference.backward(sc, ro, rd, f.color, f.others, g, go, nthreads=8)
    for mode in ("reference_arithmetic", "default"):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", reference_arithmetic=(mode != "default"))
        out = gpu_forward(tr, sc, ro, rd, st)
        grads = gpu_backward(tr, sc, ro, rd, st, out["color"], out["others"], g, go)
        tr.device_status()
        errs = {k: rel_norm(grads[k], getattr(ref, k)) for k in ("dtri", "dsigma", "dopac", "dsh")}
        print(f"{name} {mode} gradients vs the reference's code (relative L2): "
              + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
        if mode == "reference_arithmetic":
            for k, v in errs.items():
                assert v <= GRAD_RTOL, (k, v)
        else:  # the reference's own FP32 vertex gradient is the noisiest part
            for k, v in errs.items():
                assert v <= (5e-2 if k == "dtri" else 5e-3), (k, v)
