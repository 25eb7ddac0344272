"""Batched views of uneven resolution (one launch per pass), CUDA-graph replay
and the traversal autotuner, all checked against per-view calls of the same
C ABI."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, scenes  # noqa: E402
from diff_tritracer.autotune import autotune  # noqa: E402
from diff_tritracer.batch import ViewBatch  # noqa: E402
from gpu_helpers import DEV, T, rel_norm  # noqa: E402
from scenes_for_tests import dense_scene  # noqa: E402

SHAPES = [(40, 56), (24, 33), (61, 48)]  # uneven, not multiples of the 8x4 tile
ORIGINS = [(0.3, 0.4, 3.0), (-2.0, 0.5, 2.0), (0.2, -2.5, 1.5)]


def views():
    out = []
    for (H, W), o in zip(SHAPES, ORIGINS):
        cam = scenes.look_at_camera(list(o), H, W, fov_deg=12.0)
        out.append(scenes.camera_rays(cam))
    return out


def scene_tensors(sc):
    return dict(triangles_points=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), num_points_per_triangle=T(sc.num_points),
                cumsum_of_points_per_triangle=T(sc.cumsum), number_of_points=sc.P, shs=T(sc.shs),
                opacities=T(sc.opacities), scaling=torch.zeros(sc.P, device=DEV),
                density_factor=torch.zeros(sc.P, device=DEV))


def single_view(tr, s, ro, rd, g, go):
    bg = torch.zeros(3, device=DEV)
    col, oth, _, _, den, maxb = tr.trace_forward(
        T(ro), T(rd), s["triangles_points"], s["sigma"], s["num_points_per_triangle"],
        s["cumsum_of_points_per_triangle"], s["number_of_points"], s["shs"], 3, torch.empty(0, device=DEV),
        s["opacities"], torch.zeros_like(s["scaling"]), torch.zeros_like(s["density_factor"]), bg,
        torch.zeros(5, device=DEV), 0, False).data
    grads = tr.trace_backward(T(ro), T(rd), bg, s["triangles_points"], s["sigma"], s["num_points_per_triangle"],
                              s["cumsum_of_points_per_triangle"], col, oth, s["number_of_points"], s["shs"], 3,
                              s["opacities"], T(g), T(go), s["scaling"], False).data
    torch.cuda.synchronize()
    return col.cpu().numpy(), oth.cpu().numpy(), den.cpu().numpy(), maxb.cpu().numpy(), [x.cpu().numpy() for x in grads]


@pytest.mark.parametrize("traversal", ["packets", "lanes"])
def test_views_in_one_launch_match_single_views(traversal):
    sc = dense_scene(seed=6, P=3000)
    s = scene_tensors(sc)
    vs = views()
    ups = [scenes.upstream_grads(H, W, seed=i, others_std=1.0) for i, (H, W) in enumerate(SHAPES)]
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal)
    singles = [single_view(tr, s, ro, rd, g, go) for (ro, rd), (g, go) in zip(vs, ups)]
    bg = torch.zeros(3, device=DEV)
    outs, maxb = tr.trace_forward_views([(T(ro), T(rd)) for ro, rd in vs], s["triangles_points"], s["sigma"],
                                        s["num_points_per_triangle"], s["cumsum_of_points_per_triangle"],
                                        s["number_of_points"], s["shs"], 3, s["opacities"], s["scaling"],
                                        s["density_factor"], bg, 2)
    grads = tr.trace_backward_views([(T(ro), T(rd)) for ro, rd in vs], outs, [(T(g), T(go)) for g, go in ups],
                                    s["triangles_points"], s["sigma"], s["num_points_per_triangle"],
                                    s["cumsum_of_points_per_triangle"], s["number_of_points"], s["shs"], 3,
                                    s["opacities"], bg)
    torch.cuda.synchronize()
    tr.device_status()
    for (col, oth), single in zip(outs, singles):
        np.testing.assert_array_equal(col.cpu().numpy(), single[0])
        np.testing.assert_array_equal(oth.cpu().numpy(), single[1])
    np.testing.assert_array_equal(maxb.cpu().numpy(), np.max([x[3] for x in singles], axis=0))
    np.testing.assert_array_equal(s["density_factor"].cpu().numpy(), np.max([x[2] for x in singles], axis=0))
    for k in range(4):
        want = np.sum([x[4][k] for x in singles], axis=0)
        assert rel_norm(grads[k].cpu().numpy(), want) < 1e-5, k


def test_graph_replay_matches_eager():
    sc = dense_scene(seed=6, P=3000)
    vs = views()
    ups = [scenes.upstream_grads(H, W, seed=10 + i) for i, (H, W) in enumerate(SHAPES)]
    bg = torch.zeros(3, device=DEV)
    results = {}
    for graph in (True, False):
        s = scene_tensors(sc)
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
        vb = ViewBatch(tr, SHAPES, s, 3, bg, graph=graph)
        got = []
        for shift in (0.0, 0.01):  # two steps with different rays (camera moved)
            vb.set_rays([(T(ro) + shift, T(rd)) for ro, rd in vs])
            vb.set_upstream([(T(g), T(go)) for g, go in ups])
            vb.step()
            torch.cuda.synchronize()
            got.append(([c.cpu().numpy() for c, _ in vb.outputs], [g.cpu().numpy() for g in vb.grads]))
        results[graph] = got
    for (cg, gg), (ce, ge) in zip(results[True], results[False]):
        for a, b in zip(cg, ce):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(gg, ge):
            assert rel_norm(a, b) < 1e-5
    # the second step really saw the moved rays
    assert not np.array_equal(results[True][0][0][0], results[True][1][0][0])


def test_autotune_chooses_and_caches(tmp_path):
    sc = dense_scene(seed=6, P=3000)
    s = scene_tensors(sc)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    vb = ViewBatch(tr, SHAPES, s, 3, torch.zeros(3, device=DEV), graph=False)
    vb.set_rays([(T(ro), T(rd)) for ro, rd in views()])
    cache = tmp_path / "autotune.json"
    best = autotune(tr, vb.step, key="dense3000", cache_path=str(cache), iters=2)
    assert best["traversal"] in ("packets", "lanes") and cache.exists()
    from diff_tritracer.autotune import CANDIDATES

    assert len(best["all"]) == len(CANDIDATES) == 10  # 2 packet sizes x 4 forward schedules + 2 lane stacks
    again = autotune(tr, vb.step, key="dense3000", cache_path=str(cache))
    assert all(again[k] == best[k] for k in ("traversal", "k", "stack_depth", "split", "collect"))
    vb.step()
    torch.cuda.synchronize()
    tr.device_status()


def test_graph_replays_with_hit_cache_match_retraced_eager():
    """ViewBatch keeps a hit cache by default: inside the captured step the
    adjoint replays the forward's queries. Over two steps with moved vertices
    (the graph refits them) its results equal an eager batch without the cache."""
    sc = dense_scene(seed=8, P=3000)
    vs = views()
    ups = [scenes.upstream_grads(H, W, seed=20 + i, others_std=1.0) for i, (H, W) in enumerate(SHAPES)]
    bg = torch.zeros(3, device=DEV)
    rays = sum(H * W for H, W in SHAPES)
    results, replays = {}, []
    for cached in (True, False):
        s = scene_tensors(sc)
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
        vb = ViewBatch(tr, SHAPES, s, 3, bg, graph=cached, hit_cache=cached)
        vb.set_rays([(T(ro), T(rd)) for ro, rd in vs])
        vb.set_upstream([(T(g), T(go)) for g, go in ups])
        got = []
        for step in range(2):
            if step:
                s["triangles_points"].add_(0.002)  # an optimiser step, in place
            tr.reset_stats()
            vb.step()
            torch.cuda.synchronize()
            tr.device_status()
            if cached:
                replays.append(tr.stats()["hit_cache_replays"])
            got.append(([c.cpu().numpy() for c, _ in vb.outputs], [g.cpu().numpy() for g in vb.grads]))
        results[cached] = got
    assert all(n >= rays for n in replays), replays
    for (cg, gg), (ce, ge) in zip(results[True], results[False]):
        for a, b in zip(cg, ce):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(gg, ge):
            assert rel_norm(a, b) < 1e-5
    assert not np.array_equal(results[True][0][0][0], results[True][1][0][0])


def test_batch_fits_its_hit_cache_pool():
    """A batch whose cache has no pool: fit_hit_cache grows it until one
    forward's later queries all fit and records the graph again; every query
    is then replayed and the results equal an uncached eager batch."""
    sc = dense_scene(seed=8, P=3000)
    vs = views()
    ups = [scenes.upstream_grads(H, W, seed=30 + i, others_std=1.0) for i, (H, W) in enumerate(SHAPES)]
    bg = torch.zeros(3, device=DEV)
    results = {}
    for cached in (True, False):
        s = scene_tensors(sc)
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
        tr.set_traversal("packets", k=16)
        vb = ViewBatch(tr, SHAPES, s, 3, bg, graph=cached, hit_cache=cached)
        vb.set_rays([(T(ro), T(rd)) for ro, rd in vs])
        vb.set_upstream([(T(g), T(go)) for g, go in ups])
        if cached:
            vb.hit_cache = tr.new_hit_cache(vb.num_rays, pool=0)  # 16-hit queries, main part only
            vb._capture()
            vb._forward(1)
            before = tr.hit_cache_usage(vb.hit_cache)
            assert before["pool_cap"] == 0 and before["pool_used"] > 0
            use = vb.fit_hit_cache()
            assert 0 < use["pool_used"] <= use["pool_cap"]
        tr.reset_stats()
        vb.step()
        torch.cuda.synchronize()
        tr.device_status()
        st = tr.stats()
        if cached:
            assert st["hit_cache_replays"] == st["queries"]
        results[cached] = ([c.cpu().numpy() for c, _ in vb.outputs], [g.cpu().numpy() for g in vb.grads])
    for a, b in zip(results[True][0], results[False][0]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(results[True][1], results[False][1]):
        assert rel_norm(a, b) < 1e-5
