"""The CUDA path at the benchmark's full size: the seeded 1M-triangle scene
and 4 views of 800x800 (2.56M rays), the forward + adjoint workload the bench
times. The oracle cannot trace every ray in seconds, so the full-size launches
are checked through properties that do not depend on size:

* a seeded sample of 4096 pixels equals the FP64 oracle run on those rays
  alone (rays are independent), images within 1e-5 relative (+1e-6), on every
  ray whose threshold decisions are not within 1e-5 of flipping;
* the adjoint over all 2.56M rays, replaying the forward's hit cache, with
  the upstream gradient non-zero only on those sampled pixels, equals the
  oracle's adjoint of the sampled rays (gradients within 1e-4 relative);
* the traversal configurations give the same images bit for bit, a forward
  repeated gives the same bits, and the replayed adjoint equals the
  re-traversing one up to the order of float atomics (1e-6);
* the batched workload (3M triangles, 16 views of uneven size, 10.2M rays,
  one CUDA-graph replay of refit + forward + adjoint with the fitted hit
  cache): a sample of its pixels and the adjoint of that sample equal the
  oracle's.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bench import make_workload  # noqa: E402
from diff_tritracer import _C, scenes  # noqa: E402
from diff_tritracer.batch import ViewBatch  # noqa: E402
from gpu_helpers import DEV, MARGIN, T, rel_norm  # noqa: E402

P, VIEWS, H, W = 1_000_000, 4, 800, 800
N_SAMPLE = 4096
RTOL, ATOL, GRAD_RTOL = 1e-5, 1e-6, 1e-4
BG = np.array([0.1, 0.2, 0.3], np.float32)


@pytest.fixture(scope="module")
def c2():
    sc = scenes.make_scene(P, seed=0)
    rays = [scenes.camera_rays(c) for c in scenes.sphere_cameras(VIEWS, H, W, seed=0)]
    ro = np.ascontiguousarray(np.concatenate([r[0] for r in rays], 0))
    rd = np.ascontiguousarray(np.concatenate([r[1] for r in rays], 0))
    idx = np.sort(np.random.default_rng(7).choice(ro.shape[0] * ro.shape[1], N_SAMPLE, replace=False))
    dev = dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
               shs=T(sc.shs), opac=T(sc.opacities), ro=T(ro), rd=T(rd), bg=T(BG))
    sample = (ro.reshape(-1, 3)[idx][None].copy(), rd.reshape(-1, 3)[idx][None].copy())
    return sc, dev, idx, sample


def tracer(traversal, k, stack_depth=0):
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.set_traversal(traversal, k, stack_depth)
    return tr


def forward(tr, sc, d, cache=None, rebuild=0):
    res = tr.trace_forward(d["ro"], d["rd"], d["verts"], d["sigma"], d["npts"], d["cums"], sc.P, d["shs"], 3,
                           torch.empty(0, device=DEV), d["opac"], torch.zeros(sc.P, device=DEV),
                           torch.zeros(sc.P, device=DEV), d["bg"], torch.zeros(5, device=DEV), rebuild, False,
                           hit_cache=cache)
    color, others, _, scaling, density, maxb = res.data
    return color, others, scaling, density, maxb


def backward(tr, sc, d, color, others, g, go, cache=None):
    res = tr.trace_backward(d["ro"], d["rd"], d["bg"], d["verts"], d["sigma"], d["npts"], d["cums"], color, others,
                            sc.P, d["shs"], 3, d["opac"], g, go, torch.zeros(sc.P, device=DEV), False,
                            hit_cache=cache)
    return [x.cpu().numpy() for x in res.data]


def test_sampled_pixels_match_fp64_oracle(oracle, c2):
    sc, d, idx, (ro_s, rd_s) = c2
    tr = tracer("packets", 32)
    color, others = forward(tr, sc, d)[:2]
    tr.device_status()
    ref = oracle.forward(sc, ro_s, rd_s, bg=BG, precision=64, exact=True, canonical=True, record=1, nthreads=8)
    ok = ref.margin > MARGIN
    assert ok.mean() > 0.97, ok.mean()
    assert (ref.others[1, 0] > 0.5).mean() > 0.3  # the sample sees the scene
    for got, want in ((color, ref.color), (others, ref.others)):
        a = got.reshape(got.shape[0], -1)[:, idx].cpu().numpy()[:, ok]
        b = want.reshape(want.shape[0], -1)[:, ok]
        err = np.abs(a - b)
        assert np.all(err <= RTOL * np.abs(b) + ATOL), float((err / (RTOL * np.abs(b) + ATOL)).max())


def test_adjoint_of_sampled_pixels_matches_fp64_oracle(oracle, c2):
    sc, d, idx, (ro_s, rd_s) = c2
    tr = tracer("packets", 32)
    R = VIEWS * H * W
    cache = tr.new_hit_cache(R)
    color, others = forward(tr, sc, d, cache)[:2]
    ref = oracle.forward(sc, ro_s, rd_s, bg=BG, precision=64, exact=True, canonical=True, record=1, nthreads=8)
    ok = (ref.margin > MARGIN)[None, None, :]
    g_s, go_s = scenes.upstream_grads(1, N_SAMPLE, seed=9, others_std=1.0)
    g_s, go_s = g_s * ok, go_s * ok
    g = np.zeros((3, VIEWS * H, W), np.float32)
    go = np.zeros((7, VIEWS * H, W), np.float32)
    g.reshape(3, -1)[:, idx] = g_s[:, 0]
    go.reshape(7, -1)[:, idx] = go_s[:, 0]
    tr.reset_stats()
    grads = backward(tr, sc, d, color, others, T(g), T(go), cache)
    tr.device_status()
    assert tr.stats()["hit_cache_replays"] >= R
    rb = oracle.backward(sc, ro_s, rd_s, ref.color, ref.others, g_s, go_s, bg=BG, precision=64, exact=True,
                         canonical=True, nthreads=8)
    for got, key in zip(grads, ("dtri", "dsigma", "dopac", "dsh")):
        want = getattr(rb, key)
        assert np.linalg.norm(want) > 0, key
        e = rel_norm(got, want)
        assert e < GRAD_RTOL, (key, e)


def test_traversal_configurations_agree_bit_for_bit(c2):
    sc, d, _, _ = c2
    outs = []
    for cfg in (("packets", 32), ("packets", 16), ("lanes", 16, 32), ("packets", 32)):
        tr = tracer(*cfg)
        outs.append([x.cpu().numpy() for x in forward(tr, sc, d)])
        tr.device_status()
        del tr
    assert (outs[0][3] > 0).sum() > 100_000  # blended triangles
    for other in outs[1:]:  # the last one repeats the first configuration
        for a, b in zip(outs[0], other):
            np.testing.assert_array_equal(a, b)


def test_replayed_adjoint_equals_retraced(c2):
    sc, d, _, _ = c2
    tr = tracer("packets", 32)
    R = VIEWS * H * W
    g, go = scenes.upstream_grads(VIEWS * H, W, seed=3, others_std=1.0)
    g, go = T(g), T(go)
    cache = tr.new_hit_cache(R)
    tr.reset_stats()
    color, others = forward(tr, sc, d, cache)[:2]
    torch.cuda.synchronize()
    queries = tr.stats()["queries"]
    tr.reset_stats()
    replayed = backward(tr, sc, d, color, others, g, go, cache)
    assert tr.stats()["hit_cache_replays"] == queries > R
    retraced = backward(tr, sc, d, color, others, g, go, None)
    tr.device_status()
    for a, b in zip(replayed, retraced):
        assert rel_norm(a, b) < 1e-6


def test_batched_views_sample_matches_fp64_oracle(oracle):
    sc, rays, _ = make_workload("c4_3M_16views")
    shapes = [r[0].shape[:2] for r in rays]
    sizes = [h * w for h, w in shapes]
    starts = np.concatenate([[0], np.cumsum(sizes)])
    ro_all = np.concatenate([r[0].reshape(-1, 3) for r in rays])
    rd_all = np.concatenate([r[1].reshape(-1, 3) for r in rays])
    idx = np.sort(np.random.default_rng(11).choice(starts[-1], N_SAMPLE, replace=False))
    view = np.searchsorted(starts, idx, side="right") - 1
    ro_s, rd_s = ro_all[idx][None].copy(), rd_all[idx][None].copy()
    ref = oracle.forward(sc, ro_s, rd_s, precision=64, exact=True, canonical=True, record=1, nthreads=8)
    ok = ref.margin > MARGIN
    assert ok.mean() > 0.97, ok.mean()
    g_s, go_s = scenes.upstream_grads(1, N_SAMPLE, seed=13, others_std=1.0)
    g_s, go_s = g_s * ok[None, None], go_s * ok[None, None]
    ups = [(np.zeros((3, h, w), np.float32), np.zeros((7, h, w), np.float32)) for h, w in shapes]
    for j, (v, i) in enumerate(zip(view, idx)):
        y, x = divmod(int(i - starts[v]), shapes[v][1])
        ups[v][0][:, y, x] = g_s[:, 0, j]
        ups[v][1][:, y, x] = go_s[:, 0, j]
    P = sc.P
    scene = dict(triangles_points=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), num_points_per_triangle=T(sc.num_points),
                 cumsum_of_points_per_triangle=T(sc.cumsum), number_of_points=P, shs=T(sc.shs),
                 opacities=T(sc.opacities), scaling=torch.zeros(P, device=DEV), density_factor=torch.zeros(P, device=DEV))
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.set_traversal("packets", 32, 0)
    vb = ViewBatch(tr, shapes, scene, 3, torch.zeros(3, device=DEV), graph=True)
    vb.set_rays([(T(a), T(b)) for a, b in rays])
    vb.set_upstream([(T(a), T(b)) for a, b in ups])
    use = vb.fit_hit_cache()
    assert use["pool_used"] <= use["pool_cap"]
    tr.reset_stats()
    vb.step()
    torch.cuda.synchronize()
    tr.device_status()
    st = tr.stats()
    assert st["hit_cache_replays"] == st["queries"] > starts[-1]  # every query replayed
    for key, ch in (("color", 0), ("others", 1)):
        got = np.concatenate([vb.outputs[v][ch].reshape(vb.outputs[v][ch].shape[0], -1).cpu().numpy()
                              for v in range(len(shapes))], 1)[:, idx][:, ok]
        want = getattr(ref, key).reshape(got.shape[0], -1)[:, ok]
        err = np.abs(got - want)
        assert np.all(err <= RTOL * np.abs(want) + ATOL), (key, float((err / (RTOL * np.abs(want) + ATOL)).max()))
    rb = oracle.backward(sc, ro_s, rd_s, ref.color, ref.others, g_s, go_s, precision=64, exact=True, canonical=True,
                         nthreads=8)
    for got, key in zip(vb.grads, ("dtri", "dsigma", "dopac", "dsh")):
        want = getattr(rb, key)
        assert np.linalg.norm(want) > 0, key
        e = rel_norm(got.cpu().numpy(), want)
        assert e < GRAD_RTOL, (key, e)


def test_secondary_passes_sample_matches_fp64_oracle(oracle):
    """The secondary-ray passes at their benchmark configuration: 500k
    triangles, 20 % dielectric (IOR ~ U[1.3, 1.6]), a 512x1024 environment
    map, 2 views of 800x800 stacked into one [1600, 800] image, up to 2
    bounces. Pixels' ray trees are independent, so a seeded sample of 4096
    pixels of the full launch must equal the FP64 oracle's sec_radiance of
    those rays alone, and the full adjoint with the upstream gradient
    non-zero only on the sample must equal the oracle's sec_backward of the
    sample (same bars as the plain path)."""
    P3 = 500_000
    sc = scenes.make_scene(P3, seed=0)
    sec = scenes.secondary_inputs(P3, seed=0)
    cams = scenes.sphere_cameras(2, 800, 800, seed=3)
    rays = [scenes.camera_rays(c) for c in cams]
    ro = np.ascontiguousarray(np.concatenate([r[0] for r in rays], 0))
    rd = np.ascontiguousarray(np.concatenate([r[1] for r in rays], 0))
    HH, WW = ro.shape[:2]
    idx = np.sort(np.random.default_rng(17).choice(HH * WW, N_SAMPLE, replace=False))
    ro_s, rd_s = ro.reshape(-1, 3)[idx][None].copy(), rd.reshape(-1, 3)[idx][None].copy()
    ref = oracle.forward(sc, ro_s, rd_s, precision=64, exact=True, canonical=True, record=256, nthreads=8,
                         secondary=sec)
    ok = ref.margin > MARGIN
    assert ok.mean() > 0.95, ok.mean()
    g_s, go_s = scenes.upstream_grads(1, N_SAMPLE, seed=21, others_std=1.0)
    g_s, go_s = g_s * ok[None, None], go_s * ok[None, None]
    g = np.zeros((3, HH, WW), np.float32)
    go = np.zeros((7, HH, WW), np.float32)
    g.reshape(3, -1)[:, idx] = g_s[:, 0]
    go.reshape(7, -1)[:, idx] = go_s[:, 0]
    dv = dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
              shs=T(sc.shs), opac=T(sc.opacities), mat=T(sec["material"]), ior=T(sec["ior"]), env=T(sec["env"]))
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.reset_stats()
    color, others, _ = tr.trace_forward_secondary(
        T(ro), T(rd), dv["verts"], dv["sigma"], dv["npts"], dv["cums"], P3, dv["shs"], 3, dv["opac"],
        torch.zeros(P3, device=DEV), torch.zeros(P3, device=DEV), dv["mat"], dv["ior"], dv["env"], 2)
    grads = tr.trace_backward_secondary(
        T(ro), T(rd), dv["verts"], dv["sigma"], dv["npts"], dv["cums"], color, others, P3, dv["shs"], 3, dv["opac"],
        T(g), T(go), dv["mat"], dv["ior"], dv["env"], 2)
    torch.cuda.synchronize()
    tr.device_status()
    assert tr.stats()["rays"] > HH * WW * 1.2  # spawned rays went through the queue
    for got, want in ((color, ref.color), (others, ref.others)):
        a = got.reshape(got.shape[0], -1)[:, idx].cpu().numpy()[:, ok]
        b = want.reshape(want.shape[0], -1)[:, ok]
        err = np.abs(a - b)
        assert np.all(err <= RTOL * np.abs(b) + ATOL), float((err / (RTOL * np.abs(b) + ATOL)).max())
    rb = oracle.backward(sc, ro_s, rd_s, ref.color, ref.others, g_s, go_s, precision=64, exact=True, canonical=True,
                         nthreads=8, secondary=sec)
    for got, key in zip(grads, ("dtri", "dsigma", "dopac", "dsh")):
        want = getattr(rb, key)
        assert np.linalg.norm(want) > 0, key
        e = rel_norm(got.cpu().numpy(), want)
        assert e < GRAD_RTOL, (key, e)
