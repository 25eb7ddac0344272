"""Proposal network on the tensor cores (tt_mlp_*) against the numpy oracle
(oracle/proposal.py), and the learned-interval trace against the plain one.

* inference: outputs within BF16-rounding noise of the oracle, which rounds
  at the same points (inputs, weights, activations);
* training step: the kernels' weight gradients (the per-CTA sums left in the
  partial buffer) within 2 % (L2) of the oracle's, the loss within 1e-3, and
  the Adam update exact to FP32 rounding;
* training on the tracer's own records lowers the loss; on held-out views
  the far clip of the learned intervals leaves the image bit-identical to the
  plain trace (a short interval only costs a continuation); the counters
  show what the clip saves and what its continuations cost.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, proposal, scenes  # noqa: E402
from gpu_helpers import DEV, T, rel_norm  # noqa: E402
from oracle import proposal as OP  # noqa: E402


def random_rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.normal(0, 1, (n, 3))
    o = 3 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o / 3 + rng.normal(0, 0.2, (n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


@pytest.fixture(scope="module")
def tracer():
    return _C.OptixTracer("", "forward.ptx", "backward.ptx")


def make_prop(tracer, seed=3):
    p = proposal.Proposal(tracer, seed=seed, center=(0.1, -0.2, 0.05))
    # a non-trivial network: perturb the output layer and the biases too
    rng = np.random.default_rng(seed)
    m = p.master.cpu().numpy()
    W = [m[proposal.OFF[l]:proposal.OFF[l] + proposal.ROWS[l] * 80].reshape(proposal.ROWS[l], 80) for l in range(4)]
    W[0][:, 78] = rng.normal(0, 0.1, 64)
    for l in (1, 2):
        W[l][:, 64] = rng.normal(0, 0.1, 64)
    W[3][:2, :64] = rng.normal(0, 0.3, (2, 64))
    W[3][:2, 64] = [0.2, 0.6]
    p.master.copy_(torch.from_numpy(m))
    p.update()
    return p


def test_inference_matches_oracle(tracer):
    p = make_prop(tracer)
    rays = random_rays(3000, 1)  # not a multiple of the 128-ray tile
    got = p.predict(T(rays)).cpu().numpy()
    tracer.device_status()
    ref = OP.predict(p.master.cpu().numpy(), rays, p.origin_scale, p.t_shift, p.t_scale, p.center)
    err = np.abs(got - ref)
    print("inference |err| mean %.2e max %.2e, output spread %.2e" % (err.mean(), err.max(), ref.std()))
    assert ref.std() > 0.1
    assert err.mean() < 2e-3 and err.max() < 3e-2


def test_intervals_layout(tracer):
    p = make_prop(tracer)
    views = [scenes.camera_rays(scenes.look_at_camera([0.3, 0.4, 3.0], H, W, fov_deg=20.0)) for H, W in
             ((20, 24), (7, 130))]
    cap = 0.9
    ivs = p.intervals([(T(ro), T(rd)) for ro, rd in views], margin_near=0.1, margin_far=0.2, far_cap=cap)
    n_inf = n_all = 0
    for (ro, rd), iv in zip(views, ivs):
        rays = np.concatenate([ro.reshape(-1, 3), rd.reshape(-1, 3)], 1)
        raw = p.predict(T(rays)).cpu().numpy()
        s = p.offsets(T(rays)).cpu().numpy()
        got = iv.cpu().numpy().reshape(2, -1)
        np.testing.assert_allclose(got[0], raw[:, 0] - 0.1, rtol=0, atol=1e-5)
        rel = raw[:, 1] - s + 0.2  # far_cap is measured from the closest approach
        keep = np.abs(rel - cap) > 1e-4  # rounding may decide rays right at the cap either way
        want = np.where(rel >= cap, np.inf, raw[:, 1] + 0.2)
        np.testing.assert_allclose(got[1][keep], want[keep], rtol=0, atol=1e-5)
        n_inf += int(np.isinf(want).sum())
        n_all += want.size
    assert 0 < n_inf < n_all


def test_train_step_matches_oracle(tracer):
    p = make_prop(tracer)
    n = 70000  # several CTAs, a partial last tile
    rays = random_rays(n, 2)
    rng = np.random.default_rng(5)
    targets = np.stack([rng.uniform(2.0, 3.0, n), rng.uniform(3.0, 4.5, n)], 1).astype(np.float32)
    targets[::7, 0] = -1.0  # rays without hits: no t_near term
    m0 = p.master.cpu().numpy().astype(np.float64)
    loss = torch.zeros(1, device=DEV)
    p.train_step(T(rays), T(targets), lr=1e-3, near_weight=8.0, far_weight=3.0, loss_out=loss)
    torch.cuda.synchronize()
    tracer.device_status()
    ntiles = (n + 127) // 128
    per = -(-ntiles // p.partial.shape[0])
    ctas = -(-ntiles // per)
    g_gpu = p.partial[:ctas, :proposal.PARAMS].sum(0).double().cpu().numpy() / n
    l_ref, g_ref = OP.loss_and_grad(m0, rays, targets, p.origin_scale, p.t_shift, p.t_scale, 8.0, 3.0, p.center)
    e = rel_norm(g_gpu, g_ref)
    print(f"loss gpu {loss.item():.6f} oracle {l_ref:.6f}; gradient rel L2 {e:.2e}")
    assert abs(loss.item() - l_ref) <= 1e-3 * l_ref
    assert e < 2e-2
    # per layer too (the small output layer must not hide in the total)
    for l in range(4):
        sl = slice(proposal.OFF[l], proposal.OFF[l] + proposal.ROWS[l] * 80)
        assert rel_norm(g_gpu[sl], g_ref[sl]) < 3e-2, l
    # Adam, first step: m = 0.1 g, v = 0.001 g^2 -> update = lr * g / (|g| + eps / sqrt(1000)...)
    w1 = p.master.cpu().numpy().astype(np.float64)
    want, _, _ = OP.adam(m0, np.zeros_like(m0), np.zeros_like(m0), g_gpu.astype(np.float32).astype(np.float64), 1,
                         1e-3)
    np.testing.assert_allclose(w1, want, rtol=0, atol=2e-7)


def scene_dict(sc):
    return dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
                shs=T(sc.shs), opac=T(sc.opacities), P=sc.P)


def test_learned_intervals_on_tracer_records():
    """Train on the plain tracer's records of 36 views, test on 4 others."""
    # optically thick enough that many rays end on the transmittance cut-off
    sc = scenes.make_scene(20000, seed=11, center_std=0.25, edge_range=(0.06, 0.25))
    s = scene_dict(sc)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.set_work_counters(True)  # node visits and triangle tests, for the work comparison below
    tr.build_tri_accel(s["verts"], s["cums"], sc.P, True)
    cams = scenes.sphere_cameras(40, 96, 96, seed=4, fov_deg=20.0)
    views = [tuple(T(a) for a in scenes.camera_rays(c)) for c in cams]
    train, held = views[:36], views[36:]
    p = proposal.Proposal(tr, seed=0)
    rays, targets, far_target = proposal.collect(p, tr, s, train)
    p.far_target, p.far_cap = far_target, far_target - 0.25
    losses = proposal.fit(p, rays, targets, epochs=40, batch=16384, lr=3e-3)
    tr.device_status()
    first, last = losses[:5].mean(), losses[-5:].mean()
    print(f"loss {first:.4f} -> {last:.4f} over {len(losses)} steps")
    assert last < 0.2 * first
    hrays, htargets, _ = proposal.collect(p, tr, s, held, far_target=far_target)
    st = proposal.interval_stats(p, hrays, htargets)
    print("held-out", st)
    assert st["near_miss"] == 0.0  # the near clip is off by default
    assert st["terminated"] > 0.1 and st["far_clipped"] > 0.5 and st["far_err_median"] < 0.3
    bg = torch.zeros(3, device=DEV)

    def render(intervals):
        outs, _ = tr.trace_forward_views(held, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3,
                                         s["opac"], torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), bg,
                                         2, intervals=intervals)
        return torch.stack([c for c, _ in outs]).cpu().numpy()

    def work(st):  # traversal work per ray: node visits and triangle tests
        return (st["node_visits"] + st["triangle_tests"]) / st["rays"]

    tr.reset_stats()
    plain = render(None)
    st_plain = tr.stats()
    # what the clip can save at best: the plain tracer's own first / last hits
    recs = [torch.empty((3, 96, 96), device=DEV) for _ in held]
    tr.trace_forward_views(held, s["verts"], s["sigma"], s["npts"], s["cums"], sc.P, s["shs"], 3, s["opac"],
                           torch.zeros(sc.P, device=DEV), torch.zeros(sc.P, device=DEV), bg, 2, records=recs)
    perfect = [torch.stack([torch.zeros_like(r[0]), torch.where(r[2] > 0.5, r[1], torch.full_like(r[1], float("inf")))])
               for r in recs]
    tr.reset_stats()
    np.testing.assert_array_equal(render(perfect), plain)
    w_perfect = work(tr.stats())
    tr.reset_stats()
    render(p.intervals(held, margin_far=0.2))
    w_learned = work(tr.stats())
    print(f"traversal work per ray: plain {work(st_plain):.1f}, learned far clip {w_learned:.1f}, "
          f"perfect far clip {w_perfect:.1f}")
    # A far clip at each terminated ray's last visited hit saves work (the
    # k-closest queries stop there instead of collecting hits the march never
    # visits). The trained network's t_far is off by ~0.1 (median) on this
    # triangle cloud, more than the spacing of the hits past the cut-off, so
    # its clip needs a margin that gives the saving back: it may not cost
    # more than 3 % either way.
    assert w_perfect < 0.95 * work(st_plain)
    assert abs(w_learned / work(st_plain) - 1.0) < 0.03
    for mf in (0.05, 0.2):
        tr.reset_stats()
        clipped = render(p.intervals(held, margin_far=mf))
        st_clip = tr.stats()
        print(f"margin_far {mf}: node visits/ray {st_plain['node_visits'] / st_plain['rays']:.1f} -> "
              f"{st_clip['node_visits'] / st_clip['rays']:.1f}; triangle tests/ray "
              f"{st_plain['triangle_tests'] / st_plain['rays']:.1f} -> "
              f"{st_clip['triangle_tests'] / st_clip['rays']:.1f}; continuations "
              f"{st_clip['interval_continuations']}, re-traces {st_clip['interval_retraces']}")
        # the far clip never changes the result: a short interval only costs a continuation
        np.testing.assert_array_equal(clipped, plain)
    # with the near clip on, hits before t_near go missing: a small image error
    rmse = float(np.sqrt(np.mean((render(p.intervals(held, margin_near=0.05)) - plain) ** 2)))
    print(f"near clip on (margin 0.05): image RMSE {rmse:.2e}")
    tr.device_status()
