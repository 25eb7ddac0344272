"""Hit cache (tt_fwd_args.hit_cache / tt_bwd_args.hit_cache): the forward
stores every ray's k-closest queries (the first ones in the main part, later
ones in the pool while it lasts), the adjoint replays them instead of
traversing the BVH again.

* the replayed adjoint equals the re-traced one (gradients up to the order of
  float atomics) for every traversal configuration; with a pool big enough
  for every later query the adjoint replays exactly the forward's queries,
  with the default pool at least every ray's first one;
* a refit between forward and adjoint, or a different k, makes the adjoint
  ignore the cache (no replay) and still give the same gradients;
* batched views, proposed intervals and the exact adjoint replay too;
* the autograd module gives the same gradients with and without the cache;
* the forward rejects a cache smaller than tt_hit_cache_bytes;
* tt_hit_cache_usage reports the pool's capacity and demand.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import diff_tritracer  # noqa: E402
from diff_tritracer import _C, scenes  # noqa: E402
from gpu_helpers import DEV, T, rel_norm, settings  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402


def cache_bytes(k, rays, pool):
    """Hit cache layout: 32-byte header, k + 1 rows of keys a ray, k + 2 a
    pool entry, then 3k float rows of hit colours for every entry."""
    return 32 + (k + 1) * 8 * rays + (k + 2) * 8 * pool + 12 * k * (rays + pool)

H, W = 48, 64
GRAD_RTOL = 1e-6  # same hits in the same order: only the atomic summation order differs


@pytest.fixture(scope="module")
def setup():
    sc = dense_scene(seed=2, P=3000)
    ro, rd = dense_view(H=H, W=W)
    g, go = scenes.upstream_grads(H, W, seed=3, others_std=1.0)
    s = dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
             shs=T(sc.shs), opac=T(sc.opacities))
    return sc, s, T(ro), T(rd), T(g), T(go)


def forward(tr, sc, s, ro, rd, cache=None, rebuild=0):
    tr.reset_stats()
    st = settings(rebuild=rebuild)
    res = tr.trace_forward(ro, rd, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3,
                           torch.empty(0, device=DEV), s["opac"], torch.zeros(sc.P, device=DEV),
                           torch.zeros(sc.P, device=DEV), st.bg, st.extra_params, st.rebuild_gas, False,
                           hit_cache=cache)
    return res.data[0], res.data[1]


def backward(tr, sc, s, ro, rd, col, oth, g, go, cache=None):
    tr.reset_stats()
    res = tr.trace_backward(ro, rd, torch.zeros(3, device=DEV), s["verts"], s["sigma"], s["npts"], s["cums"], col,
                            oth, sc.P, s["shs"], 3, s["opac"], g, go, torch.zeros(sc.P, device=DEV), False,
                            hit_cache=cache)
    replays = tr.stats()["hit_cache_replays"]
    tr.device_status()
    return [x.cpu().numpy() for x in res.data], replays


def assert_grads_equal(a, b):
    for x, y, name in zip(a, b, ("dtri", "dsigma", "dopac", "dsh")):
        assert rel_norm(x, y) < GRAD_RTOL, name


@pytest.mark.parametrize("mode,k", [("packets", 32), ("packets", 16), ("lanes", 16)])
def test_replay_equals_retrace(setup, mode, k):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=mode)
    tr.set_traversal(mode, k=k)
    R = H * W
    cache = tr.new_hit_cache(R)
    assert cache.numel() == cache_bytes(k, R, (R + 3) // 4)
    col, oth = forward(tr, sc, s, ro, rd, cache)
    # the cache does not change the forward
    col0, oth0 = forward(tr, sc, s, ro, rd, None, rebuild=2)
    assert torch.equal(col, col0) and torch.equal(oth, oth0)
    traced, n0 = backward(tr, sc, s, ro, rd, col, oth, g, go, None)
    assert n0 == 0
    # default pool (a quarter of the rays): every first query and as many later ones as fit
    forward(tr, sc, s, ro, rd, cache, rebuild=2)  # keep: the BVH generation is unchanged
    queries = tr.stats()["queries"]
    assert queries > R  # the dense view needs later queries
    replayed, n = backward(tr, sc, s, ro, rd, col, oth, g, go, cache)
    assert R <= n <= queries
    assert_grads_equal(replayed, traced)
    # a pool for every later query: the adjoint replays exactly the forward's queries
    big = torch.empty(cache_bytes(k, R, 8 * R), dtype=torch.uint8, device=DEV)
    forward(tr, sc, s, ro, rd, big, rebuild=2)
    replayed, n = backward(tr, sc, s, ro, rd, col, oth, g, go, big)
    assert n == queries
    assert_grads_equal(replayed, traced)
    # no pool at all (the main part only): the first queries
    small = big[:cache_bytes(k, R, 0)]
    forward(tr, sc, s, ro, rd, small, rebuild=2)
    replayed, n = backward(tr, sc, s, ro, rd, col, oth, g, go, small)
    assert n == R
    assert_grads_equal(replayed, traced)


def test_stale_cache_is_ignored(setup):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal="packets")
    tr.set_traversal("packets", k=32)
    cache = tr.new_hit_cache(H * W)
    col, oth = forward(tr, sc, s, ro, rd, cache)
    traced, _ = backward(tr, sc, s, ro, rd, col, oth, g, go, None)
    # a refit after the forward: the cache may no longer match the BVH
    tr.build_tri_accel(s["verts"], s["cums"], sc.P, False)
    got, n = backward(tr, sc, s, ro, rd, col, oth, g, go, cache)
    assert n == 0
    assert_grads_equal(got, traced)
    # another k: the cache holds 32-hit queries, the adjoint now takes 16
    col, oth = forward(tr, sc, s, ro, rd, cache, rebuild=2)
    tr.set_traversal("packets", k=16)
    got, n = backward(tr, sc, s, ro, rd, col, oth, g, go, cache)
    assert n == 0
    assert_grads_equal(got, traced)


def test_views_intervals_and_exact_adjoint(setup):
    sc, s, ro, rd, g, go = setup
    views = [(ro, rd), tuple(T(a) for a in dense_view(H=7, W=130, origin=(-0.2, 0.5, 2.8)))]
    ups = [(g, go), tuple(T(a) for a in scenes.upstream_grads(7, 130, seed=4, others_std=1.0))]
    rays = sum(v[0].shape[0] * v[0].shape[1] for v in views)
    # a far clip in the middle of the cloud: unterminated rays continue beyond it
    ivs = [torch.stack([torch.zeros(v[0].shape[:2], device=DEV), torch.full(v[0].shape[:2], 2.9, device=DEV)])
           for v in views]
    for exact in (False, True):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", exact_adjoint=exact)
        tr.build_tri_accel(s["verts"], s["cums"], sc.P, True)
        for iv in (None, ivs):
            cache = tr.new_hit_cache(rays)
            outs, _ = tr.trace_forward_views(views, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3,
                                             s["opac"], torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV),
                                             torch.zeros(3, device=DEV), 2, intervals=iv, hit_cache=cache)
            res = {}
            for c in (cache, None):
                tr.reset_stats()
                gr = tr.trace_backward_views(views, outs, ups, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P,
                                             s["shs"], 3, s["opac"], torch.zeros(3, device=DEV), intervals=iv,
                                             hit_cache=c)
                res[c is None] = ([x.cpu().numpy() for x in gr], tr.stats()["hit_cache_replays"])
                tr.device_status()
            assert res[False][1] >= rays and res[True][1] == 0, (exact, iv is None)
            assert_grads_equal(res[False][0], res[True][0])


def test_autograd_module_with_and_without_cache(setup):
    sc, s, ro, rd, g, go = setup
    grads = {}
    for use in (True, False):
        tracer = diff_tritracer.Tracer(hit_cache=use)
        verts = s["verts"].clone().requires_grad_(True)
        sig, opac, shs = (s[k].clone().requires_grad_(True) for k in ("sigma", "opac", "shs"))
        color, _, _, _, others, _ = tracer(ro, rd, verts, sig, s["npts"], s["cums"], sc.P, opac,
                                           torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), shs, None,
                                           settings(rebuild=0))
        ((color * g).sum() + (others * go).sum()).backward()
        grads[use] = [x.grad.cpu().numpy() for x in (verts, sig, opac, shs)]
    assert_grads_equal(grads[True], grads[False])


def test_small_cache_rejected(setup):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")  # k = 16
    small = torch.empty(cache_bytes(16, H * W, 0) - 8, dtype=torch.uint8, device=DEV)
    with pytest.raises(RuntimeError, match="hit_cache"):
        forward(tr, sc, s, ro, rd, small)


def test_misaligned_cache_and_variant_program_rejected(setup):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    buf = tr.new_hit_cache(H * W + 8)
    with pytest.raises(RuntimeError, match="16-byte aligned"):
        forward(tr, sc, s, ro, rd, buf[8:])  # the storage is aligned, this view is not
    var = _C.OptixTracer("", "reflect.ptx", "backward.ptx")
    st = settings(rebuild=0, extra=[0.3, 0.0, 0.0, 0.0, 0.0])
    with pytest.raises(RuntimeError, match="plain program"):
        var.trace_forward(ro, rd, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3,
                          torch.empty(0, device=DEV), s["opac"], torch.zeros(sc.P, device=DEV),
                          torch.zeros(sc.P, device=DEV), st.bg, st.extra_params, st.rebuild_gas, False,
                          hit_cache=var.new_hit_cache(H * W))


def test_usage_reports_pool_capacity_and_demand(setup):
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal="packets")
    tr.set_traversal("packets", k=16)
    tr.set_collect_queries(1)  # the traversal-only pass asks for no query past a ray's cut-off
    R = H * W
    with pytest.raises(RuntimeError, match="not written by a forward"):
        tr.hit_cache_usage(torch.zeros(tr.new_hit_cache(R).numel(), dtype=torch.uint8, device=DEV))
    # a pool for every later query: the demand is exact (queries after each ray's first)
    big = tr.new_hit_cache(R, pool=8 * R)
    assert big.numel() == cache_bytes(16, R, 8 * R)
    forward(tr, sc, s, ro, rd, big)
    queries = tr.stats()["queries"]
    use = tr.hit_cache_usage(big)
    assert use == {"k": 16, "pool_cap": 8 * R, "pool_used": queries - R}
    # no pool: every ray that needs a later query asks once and is refused
    none = tr.new_hit_cache(R, pool=0)
    forward(tr, sc, s, ro, rd, none, rebuild=2)
    use = tr.hit_cache_usage(none)
    assert use["pool_cap"] == 0 and 0 < use["pool_used"] <= queries - R
    _, n = backward(tr, sc, s, ro, rd, *forward(tr, sc, s, ro, rd, none, rebuild=2), g, go, none)
    assert n == R


def test_autograd_pool_grows_to_the_later_queries(setup):
    """The autograd module starts with a pool of a quarter of the rays, reads
    what its first forwards asked for and sizes later pools to fit: from the
    third step on the adjoint replays every query."""
    sc, s, ro, rd, g, go = setup
    tracer = diff_tritracer.Tracer("forward.ptx", "backward.ptx")
    tracer.tracer.set_traversal("packets", k=16)
    opac = s["opac"].clone().requires_grad_(True)
    seen = []
    for _ in range(3):
        tracer.tracer.reset_stats()
        out = tracer(ro, rd, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, opac,
                     torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), s["shs"], None, settings())
        (out[0] * g).sum().backward()
        torch.cuda.synchronize()
        tracer.tracer.device_status()
        st = tracer.tracer.stats()
        seen.append((st["hit_cache_replays"], st["queries"]))
    assert seen[0][0] < seen[0][1], seen  # the quarter-of-the-rays pool did not hold every later query
    assert seen[2][0] == seen[2][1], seen


@pytest.mark.parametrize("collect", [1, 0], ids=["first-query", "all-queries"])
@pytest.mark.parametrize("incl", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("mode,k,sd", [("packets", 32, 0), ("packets", 16, 0), ("lanes", 16, 32), ("lanes", 16, 24)])
def test_split_forward_equals_fused(setup, mode, k, sd, incl, collect):
    """With a hit cache the forward runs as a traversal-only pass that stores
    every query and a shading pass that replays them. Its outputs equal the
    fused kernel's bit for bit, its cache serves the adjoint as well (every
    query replayed when the pool holds them all), and the gradients equal the
    fused forward's up to the order of float atomics; also with proposed
    intervals, whose continuations the shading pass traverses itself. The
    collecting pass stores each ray's first query or all of them; the
    shading pass stores the queries it traverses, so the adjoint replays
    every query of the march either way."""
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=incl, traversal=mode)
    tr.set_traversal(mode, k=k, stack_depth=sd or 32)
    tr.set_collect_queries(collect)
    R = H * W
    rng = np.random.default_rng(5)
    # intervals: a far clip inside the hits for half the rays (continuations), none for the rest
    far = np.where(rng.random((H, W)) < 0.5, 2.9, np.inf).astype(np.float32)
    iv = T(np.stack([np.zeros((H, W), np.float32), far]))
    for interval in (None, iv):
        outs = {}
        for split in (False, True):
            tr.set_split_forward(split)
            cache = tr.new_hit_cache(R, pool=4 * R)
            if interval is None:
                col, oth = forward(tr, sc, s, ro, rd, cache)
                queries = tr.stats()["queries"]
                grads, replays = backward(tr, sc, s, ro, rd, col, oth, g, go, cache)
                assert replays == queries, (split, replays, queries)
            else:
                (col, oth), = [(c, o) for c, o in tr.trace_forward_views(
                    [(ro, rd)], s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3, s["opac"],
                    torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), torch.zeros(3, device=DEV), 0,
                    intervals=[interval], hit_cache=cache)[0]]
                tr.reset_stats()
                grads = tr.trace_backward_views([(ro, rd)], [(col, oth)], [(g, go)], s["verts"], s["sigma"],
                                                s["npts"], s["cums"], sc.P, s["shs"], 3, s["opac"],
                                                torch.zeros(3, device=DEV), intervals=[interval], hit_cache=cache)
                grads = [x.cpu().numpy() for x in grads]
                replays = tr.stats()["hit_cache_replays"]
                tr.device_status()
            outs[split] = (col.cpu().numpy(), oth.cpu().numpy(), grads, replays)
        a, b = outs[False], outs[True]
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        assert_grads_equal(b[2], a[2])
        assert b[3] > 0
    tr.set_split_forward(True)


@pytest.mark.parametrize("mode,k", [("packets", 32), ("lanes", 16)])
def test_work_counters_are_opt_in(setup, mode, k):
    """Node visits and triangle tests are counted only with the option on,
    and counting changes no output."""
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=mode)
    tr.set_traversal(mode, k=k, stack_depth=32)
    outs = {}
    for on in (False, True):
        tr.set_work_counters(on)
        cache = tr.new_hit_cache(H * W, pool=4 * H * W)
        col, oth = forward(tr, sc, s, ro, rd, cache)
        st = tr.stats()
        tr.device_status()
        outs[on] = (col.cpu().numpy(), oth.cpu().numpy())
        assert st["queries"] > 0 and st["rays"] == H * W
        if on:
            assert st["node_visits"] > st["rays"] and st["triangle_tests"] > st["rays"]
            assert (st["packet_node_visits"] > 0) == (mode == "packets")
        else:
            assert st["node_visits"] == 0 and st["triangle_tests"] == 0 and st["packet_node_visits"] == 0
    np.testing.assert_array_equal(outs[False][0], outs[True][0])
    np.testing.assert_array_equal(outs[False][1], outs[True][1])


@pytest.mark.parametrize("k", [32, 16])
def test_replay_only_builds_and_their_fallback(setup, k):
    """With the first pass storing every query, the shading pass and the
    adjoint run as pairs of a replay-only build and the traversing one, and
    the device picks the traversing one when the cache is incomplete (here:
    no pool at all, so every later query was refused). Either way the image
    equals the fused forward's bit for bit and the gradients equal the
    re-traversing adjoint's."""
    sc, s, ro, rd, g, go = setup
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal="packets")
    tr.set_traversal("packets", k=k)
    R = H * W
    tr.set_split_forward(False)
    col0, oth0 = forward(tr, sc, s, ro, rd, None)
    traced, _ = backward(tr, sc, s, ro, rd, col0, oth0, g, go, None)
    tr.set_split_forward(True)
    tr.set_collect_queries(0)
    for pool in (4 * R, 0):
        cache = tr.new_hit_cache(R, pool=pool)
        col, oth = forward(tr, sc, s, ro, rd, cache, rebuild=2)
        queries = tr.stats()["queries"]
        assert torch.equal(col, col0) and torch.equal(oth, oth0), pool
        use = tr.hit_cache_usage(cache)
        assert (use["pool_used"] <= use["pool_cap"]) == (pool > 0), use
        grads, n = backward(tr, sc, s, ro, rd, col, oth, g, go, cache)
        assert n == (queries if pool > 0 else R), (pool, n, queries)
        assert_grads_equal(grads, traced)
