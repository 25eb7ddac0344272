"""Secondary-ray passes on the GPU (device ray queue: dielectric triangles
reflect and refract, an environment map lights escaping rays) against the
FP64 oracle's restatement of the same semantics (oracle.hpp sec_radiance /
sec_backward), through the C ABI:

* colour and side outputs within |d| <= 1e-5 |ref| + 1e-6 per pixel for
  every pixel whose ray tree makes no decision within 1e-5 (relative) of a
  threshold; the spawned rays are bit-identical (FP64 set-up without
  contraction on both sides);
* all four gradients within 1e-4 relative (L2);
* without dielectric triangles and with a constant environment the passes
  reproduce the plain trace with bg = that constant.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, scenes  # noqa: E402
from diff_tritracer.secondary import SecondaryTracer  # noqa: E402
from gpu_helpers import DEV, MARGIN, T, flagged_prims, rel_norm  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL = 1e-5, 1e-6
H, W = 48, 64


@pytest.fixture(scope="module")
def setup():
    sc = dense_scene(seed=7, P=3000)
    ro, rd = dense_view(H=H, W=W)
    sec = scenes.secondary_inputs(sc.P, seed=7, p_dielectric=0.3, env_shape=(32, 64), box=5)
    return sc, ro, rd, sec


def gpu_secondary(tr, sc, ro, rd, sec, g=None, go=None, max_depth=2, material_grads=False):
    color, others, maxb = tr.trace_forward_secondary(
        T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P, T(sc.shs), 3,
        T(sc.opacities), scaling := torch.zeros(sc.P, device=DEV), density := torch.zeros(sc.P, device=DEV),
        T(sec["material"]), T(sec["ior"]), T(sec["env"]), max_depth)
    out = dict(color=color, others=others, max_blending=maxb, scaling=scaling, density=density)
    if g is not None:
        out["grads"] = tr.trace_backward_secondary(
            T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), color, others, sc.P,
            T(sc.shs), 3, T(sc.opacities), T(g), T(go), T(sec["material"]), T(sec["ior"]), T(sec["env"]),
            max_depth, material_grads=material_grads)
    torch.cuda.synchronize()
    tr.device_status()
    return {k: (v.cpu().numpy() if torch.is_tensor(v) else [x.cpu().numpy() for x in v]) for k, v in out.items()}


@pytest.mark.parametrize("max_depth", [1, 2])
def test_forward_and_adjoint_vs_fp64_oracle(oracle, setup, max_depth):
    sc, ro, rd, sec = setup
    sec = dict(sec, max_depth=max_depth)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.reset_stats()
    g, go = scenes.upstream_grads(H, W, seed=11, others_std=1.0)
    ref = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=256, nthreads=8, secondary=sec)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.mean() > 0.95, ok.mean()
    g, go = g * ok[None], go * ok[None]
    got = gpu_secondary(tr, sc, ro, rd, sec, g, go, max_depth, material_grads=True)
    st = tr.stats()
    assert st["rays"] > H * W * 1.5  # the queue really held spawned rays
    for key in ("color", "others"):
        a, b = got[key][:, ok], getattr(ref, key)[:, ok]
        err = np.abs(a - b)
        worst = float((err / (RTOL * np.abs(b) + ATOL)).max())
        print(f"depth {max_depth} {key}: max abs {err.max():.2e}, worst/tol {worst:.3f}")
        assert np.all(err <= RTOL * np.abs(b) + ATOL), (key, worst)
    skip = np.zeros(sc.P, bool)
    skip[flagged_prims(ref, H, W, ok)] = True
    np.testing.assert_array_equal(got["density"][~skip], ref.density[~skip])
    np.testing.assert_allclose(got["max_blending"][~skip], ref.max_blending[~skip], rtol=RTOL, atol=ATOL)
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, precision=64, exact=True, canonical=True,
                         nthreads=8, secondary=sec)
    # the environment map's and the IOR's gradients too (the oracle's FP64
    # restatement is checked against central differences on the CPU)
    for key, x in zip(("dtri", "dsigma", "dopac", "dsh", "denv", "dior"), got["grads"]):
        e = rel_norm(x, getattr(rb, key))
        print(f"depth {max_depth} {key}: rel L2 {e:.2e}")
        assert np.linalg.norm(getattr(rb, key)) > 0
        assert e < 1e-4, (key, e)


def test_exact_adjoint_vs_fp64_oracle(oracle, setup):
    """The exact adjoint of the secondary passes (full chain rule of the
    window function, spawn geometry held constant) against the oracle's FP64
    restatement, which the CPU tests check against central differences."""
    sc, ro, rd, sec = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", exact_adjoint=True)
    g, go = scenes.upstream_grads(H, W, seed=12, others_std=1.0)
    kw = dict(precision=64, exact=True, canonical=True, nthreads=8, secondary=sec)
    ref = oracle.forward(sc, ro, rd, record=256, **kw)
    ok = (ref.margin > MARGIN).reshape(H, W)
    g, go = g * ok[None], go * ok[None]
    got = gpu_secondary(tr, sc, ro, rd, sec, g, go, 2, material_grads=True)
    rb = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, exact_adjoint=True, **kw)
    plain = oracle.backward(sc, ro, rd, ref.color, ref.others, g, go, **kw)
    assert rel_norm(rb.dtri, plain.dtri) > 1e-2  # the exact vertex gradient differs from the reference-style one
    for key, x in zip(("dtri", "dsigma", "dopac", "dsh", "denv", "dior"), got["grads"]):
        e = rel_norm(x, getattr(rb, key))
        print(f"exact {key}: rel L2 {e:.2e}")
        assert np.linalg.norm(getattr(rb, key)) > 0
        assert e < 1e-4, (key, e)


def test_reduces_to_plain(setup):
    sc, ro, rd, sec = setup
    bg = np.array([0.2, 0.4, 0.6], np.float32)
    flat = dict(sec, material=np.zeros(sc.P, np.int32), env=np.broadcast_to(bg, (4, 8, 3)).copy())
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    got = gpu_secondary(tr, sc, ro, rd, flat)
    res = tr.trace_forward(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
                           T(sc.shs), 3, torch.empty(0, device=DEV), T(sc.opacities), torch.zeros(sc.P, device=DEV),
                           torch.zeros(sc.P, device=DEV), T(bg), torch.zeros(5, device=DEV), 2, False).data
    np.testing.assert_allclose(got["color"], res[0].cpu().numpy(), rtol=1e-6, atol=1e-7)
    np.testing.assert_array_equal(got["others"], res[1].cpu().numpy())


def test_autograd_module_and_state(setup):
    sc, ro, rd, sec = setup
    mod = SecondaryTracer(max_depth=2)
    verts = T(sc.verts.reshape(-1)).requires_grad_(True)
    opac = T(sc.opacities).requires_grad_(True)
    shs = T(sc.shs).requires_grad_(True)
    sigma = T(sc.sigma).requires_grad_(True)
    args = (T(ro), T(rd), verts, sigma, T(sc.num_points), T(sc.cumsum), sc.P, opac, shs, T(sec["material"]),
            T(sec["ior"]), T(sec["env"]))
    for _ in range(2):  # build, then refit
        color, others, maxb, scaling, density = mod(*args)
        color.sum().backward()
    torch.cuda.synchronize()
    assert verts.grad.shape == verts.shape and shs.grad.shape == shs.shape
    assert torch.isfinite(shs.grad).all() and shs.grad.abs().sum() > 0
    # an adjoint without its forward is refused
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    with pytest.raises(RuntimeError, match="without a matching"):
        tr.build_tri_accel(T(sc.verts), T(sc.cumsum), sc.P, True)
        tr.trace_backward_secondary(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points),
                                    T(sc.cumsum), color.detach(), others, sc.P, T(sc.shs), 3, T(sc.opacities),
                                    torch.zeros_like(color), torch.zeros_like(others), T(sec["material"]),
                                    T(sec["ior"]), T(sec["env"]), 2)


def test_autograd_module_material_gradients(setup):
    """With the environment map and the IOR requiring gradients, the module
    returns the adjoint's material gradients for them (and the same
    geometry gradients as without)."""
    sc, ro, rd, sec = setup
    g, go = scenes.upstream_grads(H, W, seed=13, others_std=0.0)
    grads = {}
    for want in (False, True):
        mod = SecondaryTracer(max_depth=2)
        opac = T(sc.opacities).requires_grad_(True)
        env = T(sec["env"]).requires_grad_(want)
        ior = T(sec["ior"]).requires_grad_(want)
        color = mod(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P, opac,
                    T(sc.shs), T(sec["material"]), ior, env)[0]
        (color * T(g)).sum().backward()
        torch.cuda.synchronize()
        mod.tracer.device_status()
        grads[want] = (opac.grad.cpu().numpy(), env.grad, ior.grad)
    assert grads[False][1] is None and grads[False][2] is None
    _, env_g, ior_g = grads[True]
    assert env_g.shape == (32, 64, 3) and ior_g.shape == (sc.P,)
    assert env_g.abs().sum() > 0 and ior_g.abs().sum() > 0
    assert rel_norm(grads[True][0], grads[False][0]) < 1e-6


def test_adjoint_replays_the_ray_tree_queries(setup):
    """The forward stores the queries of every ray of the tree (primary rays
    in the hit cache's main part, spawned rays in its pool); the adjoint
    replays them, and gives the gradients of an adjoint that re-traverses
    (forced by a refit between the passes, which invalidates the cache)."""
    sc, ro, rd, sec = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    g, go = scenes.upstream_grads(H, W, seed=12, others_std=1.0)
    tr.reset_stats()
    fwd = gpu_secondary(tr, sc, ro, rd, sec)
    st = tr.stats()
    rays, queries = st["rays"], st["queries"]
    assert rays > H * W * 1.5 and queries > rays

    def adjoint():
        tr.reset_stats()
        gr = tr.trace_backward_secondary(
            T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), T(fwd["color"]),
            T(fwd["others"]), sc.P, T(sc.shs), 3, T(sc.opacities), T(g), T(go), T(sec["material"]), T(sec["ior"]),
            T(sec["env"]), 2)
        torch.cuda.synchronize()
        tr.device_status()
        return [x.cpu().numpy() for x in gr], tr.stats()["hit_cache_replays"]

    replayed, n = adjoint()
    print(f"pixels {H * W}, rays {rays}, queries {queries}, replayed {n}")
    assert H * W < n <= queries  # primary queries and spawned rays' queries
    if queries - H * W <= 2 * H * W:  # the pool (two entries per pixel) held every one
        assert n == queries
    tr.build_tri_accel(T(sc.verts.reshape(-1)), T(sc.cumsum), sc.P, False)  # same vertices, new generation
    traced, n0 = adjoint()
    assert n0 == 0
    for x, y, name in zip(replayed, traced, ("dtri", "dsigma", "dopac", "dsh")):
        assert rel_norm(x, y) < 1e-6, name


def test_sorted_levels_equal_spawn_order(setup):
    """Tracing each level of spawned rays in sorted order (direction octant,
    origin Morton code) changes only the schedule: the images are the same
    bit for bit and the gradients up to the order of float atomics."""
    sc, ro, rd, sec = setup
    g, go = scenes.upstream_grads(H, W, seed=13, others_std=1.0)
    outs = []
    for on in (False, True):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
        tr.set_sort_secondary(on)
        outs.append(gpu_secondary(tr, sc, ro, rd, sec, g, go, 2))
    a, b = outs
    for key in ("color", "others", "max_blending", "scaling", "density"):
        np.testing.assert_array_equal(a[key], b[key])
    for x, y, name in zip(a["grads"], b["grads"], ("dtri", "dsigma", "dopac", "dsh")):
        assert rel_norm(x, y) < 1e-6, name


def test_split_levels_equal_fused(setup):
    """With the split schedule every level is traced by a traversal-only pass
    that fills the ray tree's hit cache and a shading pass that replays it;
    the images equal the fused kernels' bit for bit and the gradients up to
    the order of float atomics, and the adjoint still replays the tree."""
    sc, ro, rd, sec = setup
    g, go = scenes.upstream_grads(H, W, seed=14, others_std=1.0)
    outs = []
    for split in (False, True):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
        tr.set_split_forward(split)
        tr.reset_stats()
        outs.append(gpu_secondary(tr, sc, ro, rd, sec, g, go, 2))
        st = tr.stats()
        outs[-1]["queries"] = st["queries"]
    a, b = outs
    for key in ("color", "others", "max_blending", "scaling", "density"):
        np.testing.assert_array_equal(a[key], b[key])
    for x, y, name in zip(a["grads"], b["grads"], ("dtri", "dsigma", "dopac", "dsh")):
        assert rel_norm(x, y) < 1e-6, name
    assert a["queries"] == b["queries"]  # the same marches, replayed or traversed
