"""Parity of the CUDA path (through the C ABI) with the oracle.

* Hit streams: the traversal's (t, primitive) sequence per ray must equal the
  oracle's BIT FOR BIT (same FP32 watertight intersector, every triangle hit in
  [0, 1000], ordered by (t, id)).
* Forward: against the FP64 oracle with exact geometry, per pixel
  |gpu - oracle| <= 1e-5 |oracle| + 1e-6 (images within 1e-5 relative), on
  every ray whose threshold decisions are not within 1e-5 (relative) of
  flipping.
* Adjoint: each gradient tensor within 1e-4 relative (L2) of the FP64 oracle
  (gradients within 1e-4 relative), with the upstream gradient of
  excluded rays set to zero so their decisions cannot matter.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # collected on CPU hosts, skipped there
    pytest.skip("needs a CUDA device", allow_module_level=True)

import diff_tritracer  # noqa: E402
from diff_tritracer import _C, scenes  # noqa: E402
from gpu_helpers import (MARGIN, DEV, T, flagged_prims, gpu_backward, gpu_forward, rel_norm,  # noqa: E402
                         settings)
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL = 1e-5, 1e-6
GRAD_RTOL = 1e-4


def cases():
    yield "dense", dense_scene(seed=1, P=3000), dense_view(H=48, W=64)
    sc = scenes.make_scene(20000, seed=5)
    cam = scenes.sphere_cameras(1, 56, 72, seed=5)[0]
    yield "random20k", sc, scenes.camera_rays(cam)


CASES = list(cases())


@pytest.fixture(scope="module")
def tracer():
    return _C.OptixTracer("", "forward.ptx", "backward.ptx")


@pytest.mark.parametrize("name,sc,rays", CASES, ids=[c[0] for c in CASES])
def test_hit_stream_bitwise(oracle, tracer, name, sc, rays):
    ro, rd = rays
    tracer.build_tri_accel(T(sc.verts), T(sc.cumsum), sc.P, True)
    ids_g, ts_g, cnt_g = [x.cpu().numpy() for x in tracer.hit_stream(T(ro), T(rd), max_hits=64)]
    tracer.device_status()
    ids_o, ts_o, cnt_o = oracle.hit_stream(sc, ro, rd, max_hits=64, nthreads=8)
    assert cnt_o.sum() > 0
    np.testing.assert_array_equal(cnt_g, cnt_o)
    n = np.minimum(cnt_o, 64)
    mask = np.arange(64)[None, :] < n[:, None]
    np.testing.assert_array_equal(ids_g[mask].astype(np.uint32), ids_o[mask])
    np.testing.assert_array_equal(ts_g[mask].view(np.uint32), ts_o[mask].view(np.uint32))


@pytest.mark.parametrize("incl", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("name,sc,rays", CASES, ids=[c[0] for c in CASES])
def test_forward_vs_fp64_oracle(oracle, name, sc, rays, incl):
    ro, rd = rays
    H, W = ro.shape[:2]
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=incl)
    bg = np.array([0.1, 0.2, 0.3], np.float32)
    st = settings(bg=bg)
    out = gpu_forward(tr, sc, ro, rd, st)
    tr.device_status()
    ref = oracle.forward(sc, ro, rd, bg=bg, precision=64, exact=True, canonical=True, tmin_inclusive=incl,
                         record=256, nthreads=8)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.mean() > 0.97, ok.mean()
    for key in ("color", "others"):
        a, b = out[key][:, ok], getattr(ref, key)[:, ok]
        err = np.abs(a - b)
        worst = float((err / (RTOL * np.abs(b) + ATOL)).max())
        print(f"{name} {key}: max abs {err.max():.2e}, worst/tol {worst:.3f}")
        assert np.all(err <= RTOL * np.abs(b) + ATOL), (key, worst)
    skip = np.zeros(sc.P, bool)
    skip[flagged_prims(ref, H, W, ok)] = True
    np.testing.assert_array_equal(out["density"][~skip], ref.density[~skip])
    np.testing.assert_allclose(out["max_blending"][~skip], ref.max_blending[~skip], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(out["scaling"][~skip], ref.scaling[~skip], rtol=1e-6, atol=1e-9)
    assert (out["density"] > 0).sum() > 100


@pytest.mark.parametrize("incl", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("name,sc,rays", CASES, ids=[c[0] for c in CASES])
def test_backward_vs_fp64_oracle(oracle, name, sc, rays, incl):
    ro, rd = rays
    H, W = ro.shape[:2]
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=incl)
    st = settings()
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, tmin_inclusive=incl, record=256,
                         nthreads=8)
    ok = (ref.margin > MARGIN).reshape(H, W)
    g, go = scenes.upstream_grads(H, W, seed=11, others_std=1.0)
    g = g * ok[None]
    go = go * ok[None]
    out = gpu_forward(tr, sc, ro, rd, st)
    grads = gpu_backward(tr, sc, ro, rd, st, out["color"], out["others"], g, go)
    tr.device_status()
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, precision=64, exact=True, canonical=True,
                         tmin_inclusive=incl, nthreads=8)
    for key in ("dtri", "dsigma", "dopac", "dsh"):
        e = rel_norm(grads[key], getattr(rb, key))
        print(f"{name} {key}: rel L2 {e:.2e}")
        assert np.linalg.norm(getattr(rb, key)) > 0
        assert e < GRAD_RTOL, (key, e)


def test_autograd_module(oracle):
    sc = dense_scene(seed=4, P=2000)
    ro, rd = dense_view(H=32, W=40)
    tr = diff_tritracer.Tracer("forward.ptx", "backward.ptx")
    verts = T(sc.verts.reshape(-1)).requires_grad_(True)  # flat [9P], as the reference's callers pass it
    sigma = T(sc.sigma).requires_grad_(True)
    opac = T(sc.opacities).requires_grad_(True)
    shs = T(sc.shs).requires_grad_(True)
    color, gpu_time, scaling, density, others, maxb = tr(
        T(ro), T(rd), verts, sigma, T(sc.num_points), T(sc.cumsum), sc.P, opac, torch.zeros(sc.P, device=DEV),
        torch.zeros(sc.P, device=DEV), shs, None, settings(debug=True))
    assert color.shape == (3, 32, 40) and others.shape == (7, 32, 40) and maxb.shape == (sc.P,)
    assert gpu_time.shape == (1,) and float(gpu_time) > 0
    g = torch.randn_like(color)
    (color * g).sum().backward()
    assert verts.grad.shape == verts.shape and sigma.grad.shape == sigma.shape
    assert opac.grad.shape == opac.shape and shs.grad.shape == shs.shape
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=128)
    np.testing.assert_allclose(color.detach().cpu().numpy(), ref.color, rtol=1e-4, atol=1e-5)


def test_refit_follows_moved_vertices(oracle):
    sc = dense_scene(seed=2, P=2500)
    ro, rd = dense_view(H=40, W=48)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    gpu_forward(tr, sc, ro, rd, settings(rebuild=0))
    rng = np.random.default_rng(0)
    moved = sc.__class__(**{**sc.__dict__})
    moved.verts = (sc.verts + rng.normal(0, 0.01, sc.verts.shape)).astype(np.float32)
    out = gpu_forward(tr, moved, ro, rd, settings(rebuild=1))  # refit
    tr.device_status()
    ids_g, ts_g, cnt_g = [x.cpu().numpy() for x in tr.hit_stream(T(ro), T(rd), max_hits=32)]
    ids_o, ts_o, cnt_o = oracle.hit_stream(moved, ro, rd, max_hits=32, nthreads=8)
    np.testing.assert_array_equal(cnt_g, cnt_o)
    ref = oracle.forward(moved, ro, rd, precision=64, exact=True, canonical=True, record=128)
    ok = ref.margin > MARGIN
    a, b = out["color"].reshape(3, -1)[:, ok], ref.color.reshape(3, -1)[:, ok]
    assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL)
    # keep: same structure again
    out2 = gpu_forward(tr, moved, ro, rd, settings(rebuild=2))
    np.testing.assert_array_equal(out2["color"], out["color"])


@pytest.mark.parametrize("P", [1, 2, 3, 5, 17])
def test_tiny_scenes(oracle, P):
    sc = scenes.make_scene(P, seed=P, center_std=0.02, edge_range=(0.3, 0.5))
    cam = scenes.look_at_camera([0.0, 0.2, 3.0], 24, 24, fov_deg=20.0)
    ro, rd = scenes.camera_rays(cam)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    out = gpu_forward(tr, sc, ro, rd, settings())
    tr.device_status()
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=64)
    ok = ref.margin > MARGIN
    a, b = out["color"].reshape(3, -1)[:, ok], ref.color.reshape(3, -1)[:, ok]
    assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL)


def test_rays_missing_everything(oracle):
    sc = dense_scene(seed=1, P=500)
    cam = scenes.look_at_camera([0.0, 0.0, 3.0], 16, 16, fov_deg=10.0, target=(0.0, 0.0, 10.0))
    ro, rd = scenes.camera_rays(cam)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    bg = np.array([0.25, 0.5, 0.75], np.float32)
    out = gpu_forward(tr, sc, ro, rd, settings(bg=bg))
    np.testing.assert_array_equal(out["color"], np.broadcast_to(bg[:, None, None], (3, 16, 16)))
    assert np.all(out["others"] == 0)
    assert np.all(out["max_blending"] == 0)


def test_invalid_arguments_raise():
    sc = dense_scene(seed=1, P=100)
    ro, rd = dense_view(H=8, W=8)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    with pytest.raises(RuntimeError, match="sh_degree"):
        gpu_forward(tr, sc, ro, rd, settings(sh_degree=4))
    with pytest.raises(RuntimeError, match="rebuild_gas=2 before"):
        gpu_forward(_C.OptixTracer(), sc, ro, rd, settings(rebuild=2))
    with pytest.raises(RuntimeError, match="float32"):
        tr.trace_forward(T(ro).double(), T(rd), T(sc.verts), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
                         T(sc.shs), 3, torch.empty(0, device=DEV), T(sc.opacities), torch.zeros(sc.P, device=DEV),
                         torch.zeros(sc.P, device=DEV), torch.zeros(3, device=DEV), torch.zeros(5, device=DEV), 0,
                         False)
    with pytest.raises(Exception, match="excatly one"):
        diff_tritracer.Tracer()(T(ro), T(rd), T(sc.verts), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
                                T(sc.opacities), None, None, None, None, settings())


@pytest.mark.parametrize("name,sc,rays", CASES, ids=[c[0] for c in CASES])
def test_traversal_modes_agree(name, sc, rays):
    """Warp packets and independent lanes walk the same hit stream: identical
    forward outputs bit for bit, gradients equal up to atomic summation order."""
    ro, rd = rays
    H, W = ro.shape[:2]
    g, go = scenes.upstream_grads(H, W, seed=5, others_std=1.0)
    outs = {}
    for mode in ("packets", "lanes"):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=mode)
        f = gpu_forward(tr, sc, ro, rd, settings())
        b = gpu_backward(tr, sc, ro, rd, settings(), f["color"], f["others"], g, go)
        tr.device_status()
        outs[mode] = (f, b)
    (fp, bp), (fl, bl) = outs["packets"], outs["lanes"]
    for k in ("color", "others", "max_blending", "density", "scaling"):
        np.testing.assert_array_equal(fp[k], fl[k], err_msg=k)
    for k in ("dtri", "dsigma", "dopac", "dsh"):
        assert rel_norm(bp[k], bl[k]) < 1e-5, k


VARIANTS = [("reflect.ptx", 1), ("refract.ptx", 2), ("envlight.ptx", 3)]


@pytest.mark.parametrize("prog,variant", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_sphere_variants_vs_fp64_oracle(oracle, prog, variant):
    """Reflect / refract / envlight programs (forward only, as in the
    reference) against the FP64 oracle's restatement of reflect.cu,
    refract.cu and envlight.cu. The bent rays are built with the same FP32
    operations on both sides; envlight's sample directions go through cosf /
    sinf, whose last-bit differences between CUDA and the host libm move the
    sample rays slightly, so its tolerance is wider."""
    from scenes_for_tests import sphere_extra

    sc = dense_scene(seed=1, P=3000)
    ro, rd = dense_view(H=48, W=64)
    H, W = ro.shape[:2]
    extra = sphere_extra(samples=3)
    bg = np.array([0.1, 0.2, 0.3], np.float32)
    tr = _C.OptixTracer("", prog, "backward.ptx")
    out = gpu_forward(tr, sc, ro, rd, settings(bg=bg, extra=extra))
    tr.device_status()
    ref = oracle.forward(sc, ro, rd, bg=bg, extra=extra, variant=variant, precision=64, exact=True,
                         canonical=True, record=512, nthreads=8)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.mean() > 0.9
    plain = oracle.forward(sc, ro, rd, bg=bg, precision=64, exact=True, canonical=True, nthreads=8)
    assert (np.abs(ref.color - plain.color).max(0) > 1e-4).mean() > 0.2  # the sphere bends many rays
    err = np.abs(out["color"] - ref.color)[:, ok]
    b = np.abs(ref.color)[:, ok]
    print(f"{prog}: max abs {err.max():.2e}, rms {np.sqrt((err ** 2).mean()):.2e}")
    assert np.all(out["others"] == 0)
    if variant == 3:
        assert np.sqrt((err ** 2).mean()) < 1e-4 and err.max() < 2e-2
    else:
        assert np.all(err <= RTOL * b + ATOL)
    # reference-style backward after a variant forward: the plain adjoint
    g, go = scenes.upstream_grads(H, W, seed=3)
    grads = gpu_backward(tr, sc, ro, rd, settings(bg=bg), out["color"], out["others"], g, go)
    assert all(np.isfinite(v).all() for v in grads.values())


@pytest.mark.parametrize("traversal", ["packets", "lanes"])
def test_exact_adjoint_vs_fp64_oracle(oracle, traversal):
    """exact_adjoint=True: the forward accumulates depth, middepth and
    distortion and the adjoint is the full chain rule (checked against finite differences on the CPU oracle in
    test_oracle_fd.py); the GPU's FP32 evaluation against the FP64 oracle."""
    sc, (ro, rd) = dense_scene(seed=1, P=3000), dense_view(H=48, W=64)
    H, W = ro.shape[:2]
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal, exact_adjoint=True)
    kw = dict(precision=64, exact=True, canonical=True, nthreads=8, exact_adjoint=True)
    ref = oracle.forward(sc, ro, rd, record=256, **kw)
    ok = (ref.margin > MARGIN).reshape(H, W)
    g, go = scenes.upstream_grads(H, W, seed=12, others_std=1.0)
    go[5:7] = np.random.default_rng(12).normal(0, 1.0, (2, H, W))  # middepth, distortion
    g, go = g * ok[None], go * ok[None]
    out = gpu_forward(tr, sc, ro, rd, settings())
    assert np.abs(out["others"][0]).max() > 1.0  # depth is accumulated
    assert out["others"][5].max() > 1.0 and out["others"][6].max() > 0  # middepth, distortion
    a, b = out["others"][:, ok], ref.others[:, ok]
    assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL)
    grads = gpu_backward(tr, sc, ro, rd, settings(), out["color"], out["others"], g, go)
    tr.device_status()
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, **kw)
    for key, tol in (("dtri", 1e-3), ("dsigma", GRAD_RTOL), ("dopac", GRAD_RTOL), ("dsh", GRAD_RTOL)):
        e = rel_norm(grads[key], getattr(rb, key))
        print(f"exact {traversal} {key}: rel L2 {e:.2e}")
        assert e < tol, (key, e)
    # and it differs from the reference's partial vertex gradient
    plain = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal)
    pout = gpu_forward(plain, sc, ro, rd, settings())
    pg = gpu_backward(plain, sc, ro, rd, settings(), pout["color"], pout["others"], g, go)
    assert rel_norm(pg["dtri"], grads["dtri"]) > 0.1


def test_colors_precomp_vs_fp64_oracle(oracle):
    """shs empty + colors_precomp [P, 3]: the colours replace SH (the
    reference accepts the tensor and never reads it), with their gradient."""
    sc, (ro, rd) = dense_scene(seed=3, P=3000), dense_view(H=40, W=56)
    H, W = ro.shape[:2]
    cols = np.random.default_rng(8).uniform(0.0, 1.0, (sc.P, 3)).astype(np.float32)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    empty = torch.empty(0, device=DEV)
    res = tr.trace_forward(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
                           empty, 3, T(cols), T(sc.opacities), torch.zeros(sc.P, device=DEV),
                           torch.zeros(sc.P, device=DEV), torch.zeros(3, device=DEV), torch.zeros(5, device=DEV), 0,
                           False).data
    color, others = res[0], res[1]
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=256, nthreads=8, precomp=cols)
    ok = (ref.margin > MARGIN).reshape(H, W)
    a, b = color.cpu().numpy()[:, ok], ref.color[:, ok]
    assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL)
    g, go = scenes.upstream_grads(H, W, seed=13, others_std=1.0)
    g, go = g * ok[None], go * ok[None]
    bres = tr.trace_backward(T(ro), T(rd), torch.zeros(3, device=DEV), T(sc.verts.reshape(-1)), T(sc.sigma),
                             T(sc.num_points), T(sc.cumsum), color, others, sc.P, empty, 3, T(sc.opacities), T(g), T(go),
                             torch.zeros(sc.P, device=DEV), False, colors_precomp=T(cols))
    torch.cuda.synchronize()
    tr.device_status()
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, precision=64, exact=True, canonical=True,
                         nthreads=8, precomp=cols)
    assert rel_norm(bres.dL_dcolors.cpu().numpy(), rb.dcolors) < GRAD_RTOL
    for key, x in zip(("dtri", "dsigma", "dopac"), bres.data[:3]):
        assert rel_norm(x.cpu().numpy(), getattr(rb, key)) < GRAD_RTOL, key
    # through the drop-in module: shs=None, colors_precomp given
    cp = T(cols).requires_grad_(True)
    tracer = diff_tritracer.Tracer("forward.ptx", "backward.ptx")
    out = tracer(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
                 T(sc.opacities), torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), None, cp, settings())
    (out[0] * T(g)).sum().backward()
    torch.cuda.synchronize()
    assert cp.grad is not None and rel_norm(cp.grad.cpu().numpy(), rb.dcolors) < GRAD_RTOL


def test_bvh_save_and_load(tmp_path):
    """A saved BVH topology, loaded into a fresh handle (refitted to the same
    or to moved vertices), traces exactly like the original structure."""
    sc = dense_scene(seed=2, P=2500)
    ro, rd = dense_view(H=32, W=40)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.build_tri_accel(T(sc.verts), T(sc.cumsum), sc.P, True)
    path = tmp_path / "scene.bvh"
    blob = tr.save_bvh(str(path))
    assert path.stat().st_size == len(blob) > 0
    ref = [x.cpu().numpy() for x in tr.hit_stream(T(ro), T(rd), max_hits=48)]
    tr2 = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr2.load_bvh(str(path), T(sc.verts), T(sc.cumsum), sc.P)
    got = [x.cpu().numpy() for x in tr2.hit_stream(T(ro), T(rd), max_hits=48)]
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    out1 = gpu_forward(tr, sc, ro, rd, settings(rebuild=2))
    out2 = gpu_forward(tr2, sc, ro, rd, settings(rebuild=2))
    np.testing.assert_array_equal(out1["color"], out2["color"])
    # loading onto moved vertices equals refitting the original
    moved = sc.__class__(**{**sc.__dict__})
    moved.verts = (sc.verts + np.random.default_rng(1).normal(0, 0.005, sc.verts.shape)).astype(np.float32)
    tr.build_tri_accel(T(moved.verts), T(moved.cumsum), moved.P, False)  # refit
    tr3 = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr3.load_bvh(blob, T(moved.verts), T(moved.cumsum), moved.P)
    a = [x.cpu().numpy() for x in tr.hit_stream(T(ro), T(rd), max_hits=48)]
    b = [x.cpu().numpy() for x in tr3.hit_stream(T(ro), T(rd), max_hits=48)]
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    tr3.device_status()
    with pytest.raises(RuntimeError, match="not a BVH blob"):
        _C.OptixTracer("", "forward.ptx", "backward.ptx").load_bvh(blob, T(sc.verts[:100]), T(sc.cumsum[:100]), 100)
