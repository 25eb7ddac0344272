"""Benchmark: forward+backward Mrays/s of the differentiable k-closest-hit
triangle tracer on one node.

Workload (default): 1M triangles from the seeded synthetic generator, 4 views
of 800x800 on a radius-3 sphere, stacked into one [3200, 800] ray array, fp32,
forward + backward with upstream dL/dcolor ~ N(0, 1). One step = BVH refit +
forward trace + adjoint trace (what one optimiser step of the caller runs).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0). Multi-GPU runs are independent replicas (the
tracer does not shard; each rank traces its own copy of the workload) and
report the aggregate with the max time over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "diff-triangle-tracer_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "fwd+bwd Mrays/s, proposal vs plain on B200 at RMSE≤1e-3; vs OptiX ref"
WORKLOADS = {
    # name: (triangles, views, H, W)
    "c2_1M_4x800": (1_000_000, 4, 800, 800),
    "c1_100k_1x400": (100_000, 1, 400, 400),
    # one view of the 1M scene: the profiling case (inputs still larger than L2)
    "c2_1M_1x800": (1_000_000, 1, 800, 800),
    # 16 views of uneven resolution over 3M triangles, one graph-captured launch per pass
    "c4_3M_16views": (3_000_000, 16, 0, 0),
}
C4_SIDES = (256, 512, 768, 1024)


def scenes_module():
    """The seeded scene generator (diff_tritracer/scenes.py), loaded from its
    file. It needs only numpy; importing it through the package would run the
    package's __init__, which loads the tracer library, and the reference arm
    must not map that library."""
    import importlib.util

    name = "_tt_bench_scenes"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(PKG, "diff_tritracer", "scenes.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def c4_views(seed=0):
    """16 cameras on the radius-3 sphere, side lengths drawn from {256, 512, 768, 1024}."""
    scenes = scenes_module()

    rng = np.random.default_rng(seed + 4)
    sides = rng.choice(C4_SIDES, size=16)
    cams = [scenes.sphere_cameras(1, int(n), int(n), seed=seed + 100 + i)[0] for i, n in enumerate(sides)]
    return [scenes.camera_rays(c) for c in cams]


def make_workload(name, seed=0):
    scenes = scenes_module()

    P, views, H, W = WORKLOADS[name]
    sc = scenes.make_scene(P, seed=seed)
    if name.startswith("c4"):
        rays = c4_views(seed)
        ups = [scenes.upstream_grads(r[0].shape[0], r[0].shape[1], seed=seed + i) for i, r in enumerate(rays)]
        return sc, rays, ups
    cams = scenes.sphere_cameras(views, H, W, seed=seed)
    rays = [scenes.camera_rays(c) for c in cams]
    ro = np.ascontiguousarray(np.concatenate([r[0] for r in rays], 0))
    rd = np.ascontiguousarray(np.concatenate([r[1] for r in rays], 0))
    g, go = scenes.upstream_grads(ro.shape[0], ro.shape[1], seed=seed)
    return sc, ro, rd, g, go


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: have it sampling before the
            # timed region begins, so that short regions still get samples
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.first = len(self.lines)
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return None
        # a region shorter than the sampling period: the next sample, taken as it ends
        t0 = time.time()
        while len(self.lines) <= self.first and time.time() - t0 < 0.5 and self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        time.sleep(0.05)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def sample_rows(H, n):
    """n rows spread evenly over all H rows of the stacked views (every view
    contributes in proportion to its height)."""
    n = int(max(1, min(H, n)))
    return (np.arange(n, dtype=np.int64) * H) // n + (H // n) // 2


def row_sample(ro, rd, g, go, idx):
    """The rays and upstream gradients of the sampled rows, as one image."""
    c = np.ascontiguousarray
    return c(ro[idx]), c(rd[idx]), c(g[:, idx]), c(go[:, idx])


def cpu_run(runner, sc, sample, nthreads):
    """One forward + backward of the CPU implementation over a row sample."""
    ro, rd, g, go = sample
    f = runner.forward(sc, ro, rd, nthreads=nthreads)
    runner.backward(sc, ro, rd, f.color, f.others, g, go, nthreads=nthreads)


def cpu_baseline(name, sc, ro, rd, g, go, budget_s=12.0):
    """Times the reference's own per-ray code built for the host (oracle/_ref)
    if it was built, else the oracle's FP32 port, on all host cores, over a
    bounded sample of rows spread evenly across all stacked views."""
    from oracle import pyoracle

    if pyoracle.reference_available():
        runner, kind = pyoracle.Reference(), "reference"
    else:
        runner, kind = pyoracle.Oracle(), "port"
    nthreads = os.cpu_count() or 1
    H, W = ro.shape[:2]  # the views stacked vertically
    view_h = WORKLOADS[name][2]
    t0 = time.time()
    runner._scene(sc)  # CPU BVH over the same triangles (not timed)
    build_s = time.time() - t0

    # the host code deals whole rows to its threads in turn: the probe gives
    # every thread two rows, and the sample is rescaled until it fills at
    # least half the budget (or holds every row)
    n = 2 * nthreads
    for _ in range(3):
        sample = row_sample(ro, rd, g, go, sample_rows(H, n))
        t0 = time.time()
        cpu_run(runner, sc, sample, nthreads)
        dt = max(time.time() - t0, 1e-3)
        if dt >= 0.5 * budget_s or n >= H:
            break
        n = int(min(H, n * budget_s / dt))
    n = sample[0].shape[0]
    reps = 1
    if dt < 0.5 * budget_s:  # every row is in the sample: repeat whole passes
        reps = int(np.ceil(budget_s / dt))
        t0 = time.time()
        for _ in range(reps):
            cpu_run(runner, sc, sample, nthreads)
        dt = time.time() - t0
    nrays = n * W
    runner.close()
    return {"value": reps * nrays / dt / 1e6, "unit": "Mrays/s", "cores": nthreads, "kind": kind,
            "sample": f"{n} of the {H} rows of the {H // view_h} stacked {view_h}-row views, spread evenly "
                      f"over all views ({nrays} rays, fwd+bwd) x {reps}, {dt:.1f} s; CPU BVH build "
                      f"{build_s:.1f} s untimed"}, \
        runner, kind, nthreads, sample


def slowest_rank_ms(ms, world, dev):
    """Device time of the timed region on the slowest rank. Every rank calls
    this with its own CUDA-event time, at the same point: it is the only
    collective of the replicas, which share no data."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(ms)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_arm(args, rank):
    if rank != 0:
        return
    name = args.workload
    sc, ro, rd, g, go = make_workload(name)
    base, runner, kind, nthreads, sample = cpu_baseline(name, sc, ro, rd, g, go, budget_s=args.ref_budget)
    from oracle import pyoracle

    runner = pyoracle.Reference() if kind == "reference" else pyoracle.Oracle()
    runner._scene(sc)
    for _ in range(args.warmup):
        cpu_run(runner, sc, sample, nthreads)
    times = []
    for _ in range(args.steps):
        t0 = time.time()
        cpu_run(runner, sc, sample, nthreads)
        times.append(time.time() - t0)
    nrays = sample[0].shape[0] * sample[0].shape[1]
    total = sum(times)
    value = nrays * args.steps / total / 1e6
    P, views, H, W = WORKLOADS[name]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "triangles": P, "views": views, "H": H, "W": W,
                   "rays_per_step": views * H * W, "sample_rays_per_step": nrays,
                   "sample": "rows spread evenly over all views of the workload; Mrays/s of the sample",
                   "step": "forward + adjoint of the reference's per-ray code on the host cores"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": nthreads, "kind": kind,
                         "sample": base["sample"]},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def algorithmic_bytes(rays, evals, blends, cache_k=0, colors=False):
    """Per launch, from the per-ray figures: forward 24 + 40 + 48 h_e + 204 h_b;
    adjoint 24 + 40 + 28 + 48 h_e + (192 + 2*236) h_b (h_e/h_b = evaluated /
    blended hits, counted by the forward kernel); with a hit cache of k-hit
    queries, (k + 1) * 8 bytes per ray more: written by the forward, read by
    the adjoint. With the hit colours in the cache (warp-packet traversals),
    the forward writes 12 bytes a blended hit and the adjoint reads those 12
    instead of its 192 bytes of SH."""
    c = (cache_k + 1) * 8 if cache_k else 0
    col = 12 if (cache_k and colors) else 0
    fwd = rays * (24 + 40 + c) + 48 * evals + (204 + col) * blends
    bwd = rays * (24 + 40 + 28 + c) + 48 * evals + ((12 if col else 192) + 2 * 236) * blends
    return fwd, bwd


def proposal_leg(dev, steps=3, seed=0, small=False, epochs=120):
    """The learned proposal against the plain traversal on the 3M-triangle
    workload: 64 training views of 256x256 (4.2M rays traced by the plain
    tracer), Adam on the tensor-core kernels, then forward + adjoint of 8
    held-out 1920x1080 views (one batched launch each) with and without the
    proposal's intervals, and with the perfect intervals of the plain
    tracer's own hit records (the clip's upper bound).

    Choices made on 2 validation views (other cameras than the 8 test views,
    same resolution): the far margin, the forward's schedule (fused, or split
    storing first / all queries), and whether a near clip is used (only if its
    image RMSE and gradient error against the plain trace stay <= 1e-3 there).
    Each arm is then timed on the test views under its own best schedule."""
    import time

    import torch

    from diff_tritracer import _C, proposal, scenes

    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    # small: the same protocol at profiling size (200k triangles, 16 x 128^2 training views, 2 x 540x960)
    P, n_train, side, n_held, hh, ww = (200_000, 16, 128, 2, 540, 960) if small else (3_000_000, 64, 256, 8, 1080, 1920)
    sc = scenes.make_scene(P, seed=seed)
    S = dict(verts=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), npts=T(sc.num_points), cums=T(sc.cumsum),
             shs=T(sc.shs), opac=T(sc.opacities), P=sc.P)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.set_traversal("packets", 32)
    tr.build_tri_accel(S["verts"], S["cums"], sc.P, True)
    train = [tuple(T(a) for a in scenes.camera_rays(c))
             for c in scenes.sphere_cameras(n_train, side, side, seed=1000)]
    held = [tuple(T(a) for a in scenes.camera_rays(c)) for c in scenes.sphere_cameras(n_held, hh, ww, seed=2000)]
    ups = [tuple(T(a) for a in scenes.upstream_grads(hh, ww, seed=3000 + i)) for i in range(n_held)]
    val = [tuple(T(a) for a in scenes.camera_rays(c)) for c in scenes.sphere_cameras(2, hh, ww, seed=4000)]
    val_ups = [tuple(T(a) for a in scenes.upstream_grads(hh, ww, seed=5000 + i)) for i in range(2)]
    bg = torch.zeros(3, device=dev)
    R = sum(ro.shape[0] * ro.shape[1] for ro, _ in held)

    def fwd_bwd(views, upstream, intervals, records=None):
        z1, z2 = torch.zeros(sc.P, device=dev), torch.zeros(sc.P, device=dev)
        rays = sum(ro.shape[0] * ro.shape[1] for ro, _ in views)
        cache = tr.new_hit_cache(rays)  # both arms replay the forward's queries in the adjoint
        outs, _ = tr.trace_forward_views(views, S["verts"], S["sigma"], S["npts"], S["cums"], sc.P, S["shs"], 3,
                                         S["opac"], z1, z2, bg, 2, intervals=intervals, records=records,
                                         hit_cache=cache)
        g = tr.trace_backward_views(views, outs, upstream, S["verts"], S["sigma"], S["npts"], S["cums"], sc.P,
                                    S["shs"], 3, S["opac"], bg, intervals=intervals, hit_cache=cache)
        return outs, g

    def timed(fn, n=steps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    schedules = (("fused", False, 1), ("split_first", True, 1), ("split_two", True, 2), ("split_all", True, 0))

    def set_schedule(name):
        _, split, collect = next(x for x in schedules if x[0] == name)
        tr.set_split_forward(split)
        tr.set_collect_queries(collect)

    def by_schedule(fn, n=steps):
        out = {}
        for name, _, _ in schedules:
            set_schedule(name)
            out[name] = timed(fn, n)
        return out

    def best(d):
        k = min(d, key=d.get)
        return k, d[k]

    # ---- plain arm and the perfect intervals (plain tracer's own records)
    ms_plain_modes = by_schedule(lambda: fwd_bwd(held, ups, None))
    plain_sched, ms_plain = best(ms_plain_modes)
    set_schedule(plain_sched)
    recs = [torch.empty((3, ro.shape[0], ro.shape[1]), device=dev) for ro, _ in held]
    ref_outs, ref_g = fwd_bwd(held, ups, None, recs)
    ref_col = torch.stack([c for c, _ in ref_outs]).clone()
    ref_g = [x.clone() for x in ref_g]
    perfect = [torch.stack([torch.where(torch.isfinite(r[0]), r[0], torch.zeros_like(r[0])),
                            torch.where(r[2] > 0.5, r[1], torch.full_like(r[1], float("inf")))]) for r in recs]
    perfect_far = [torch.stack([torch.zeros_like(p[0]), p[1]]) for p in perfect]
    ms_perfect = best(by_schedule(lambda: fwd_bwd(held, ups, perfect)))[1]
    ms_perfect_far = best(by_schedule(lambda: fwd_bwd(held, ups, perfect_far)))[1]

    # ---- training
    center = tuple(float(x) for x in sc.verts.reshape(-1, 3).mean(0))
    prop = proposal.Proposal(tr, seed=seed, center=center)
    t0 = time.time()
    rays, targets, far_target = proposal.collect(prop, tr, S, train)
    torch.cuda.synchronize()
    t_collect = time.time() - t0
    prop.far_target, prop.far_cap = far_target, far_target - 0.75
    t0 = time.time()
    losses = proposal.fit(prop, rays, targets, epochs=epochs, batch=65536, lr=1e-3)
    torch.cuda.synchronize()
    t_fit = time.time() - t0
    n_steps = len(losses)

    # ---- choices on the validation views
    set_schedule("fused")
    val_out, val_g = fwd_bwd(val, val_ups, None)
    val_col = torch.stack([c for c, _ in val_out]).clone()
    val_g = [x.clone() for x in val_g]
    choices = {}
    for mf in (0.1, 0.2, 0.3, 0.5, 0.75):
        ivs = prop.intervals(val, margin_near=proposal.NO_NEAR_CLIP, margin_far=mf)
        for name, ms in by_schedule(lambda: fwd_bwd(val, val_ups, ivs), n=2).items():
            choices[(mf, name, "off")] = ms
    mf_best, sched_best, _ = min(choices, key=choices.get)
    near_eval = {}
    for mn in (0.5, 0.25):
        ivs = prop.intervals(val, margin_near=mn, margin_far=mf_best)
        set_schedule(sched_best)
        outs, g = fwd_bwd(val, val_ups, ivs)
        col = torch.stack([c for c, _ in outs])
        rmse = float(((col - val_col) ** 2).mean().sqrt())
        gerr = max(float((a - b).norm() / b.norm()) for a, b in zip(g, val_g))
        ms = timed(lambda: fwd_bwd(val, val_ups, ivs), n=2)
        near_eval[mn] = {"rmse": rmse, "grad_rel_err": gerr, "ms": ms}
        if rmse <= 1e-3 and gerr <= 1e-3:
            choices[(mf_best, sched_best, mn)] = ms
    mf_best, sched_best, near = min(choices, key=choices.get)
    prop.margin_far = mf_best
    prop.margin_near = proposal.NO_NEAR_CLIP if near == "off" else near

    # ---- the learned arm on the test views
    ivs = prop.intervals(held)
    ms_infer = timed(lambda: prop.intervals(held, out=ivs))
    ms_prop_modes = by_schedule(lambda: fwd_bwd(held, ups, ivs))
    prop_sched, ms_prop = best(ms_prop_modes)
    set_schedule(prop_sched)
    tr.reset_stats()
    outs, g = fwd_bwd(held, ups, ivs)
    st = tr.stats()
    tr.device_status()
    col = torch.stack([c for c, _ in outs])
    rmse = float(((col - ref_col) ** 2).mean().sqrt())
    grad_rel = max(float((a - b).norm() / b.norm()) for a, b in zip(g, ref_g))
    hr, ht, _ = proposal.collect(prop, tr, S, held[:2], far_target=far_target)
    stats = proposal.interval_stats(prop, hr, ht)
    tr.set_split_forward(True)
    tr.set_collect_queries(1)
    flops_ray = 2 * (3 * 80 * 64 + 80 * 16)
    return {
        "workload": f"{P} triangles; train {n_train} views {side}x{side} ({int(rays.shape[0])} rays); "
                    f"test {n_held} held-out views {ww}x{hh}; margins and schedule chosen on 2 other views",
        "plain_mrays": R / ms_plain / 1e3,
        "proposal_mrays": R / (ms_prop + ms_infer) / 1e3,
        "speedup": ms_plain / (ms_prop + ms_infer),
        "schedule": {"plain": plain_sched, "proposal": prop_sched},
        "mrays_by_schedule": {"plain": {k: R / v / 1e3 for k, v in ms_plain_modes.items()},
                              "proposal": {k: R / (v + ms_infer) / 1e3 for k, v in ms_prop_modes.items()}},
        "perfect_interval_mrays": R / ms_perfect / 1e3,
        "perfect_far_only_mrays": R / ms_perfect_far / 1e3,
        "image_rmse_vs_plain": rmse, "grad_rel_err_vs_plain": grad_rel,
        "intervals": {k: round(v, 4) for k, v in stats.items()},
        "continuations_per_ray": st["interval_continuations"] / max(st["rays"], 1),
        "margin_far": prop.margin_far, "far_cap": prop.far_cap,
        "near_clip": "off" if near == "off" else f"margin {near}",
        "validation": {"ms": {f"far {k[0]} / {k[1]} / near {k[2]}": v for k, v in choices.items()},
                       "near_clip": {str(k): v for k, v in near_eval.items()}},
        "train": {"steps": n_steps, "epochs": epochs, "batch": 65536, "lr": 1e-3, "seconds": t_fit,
                  "collect_s": t_collect, "loss_first": float(losses[:5].mean()),
                  "loss_last": float(losses[-5:].mean()),
                  "tflops": 3 * flops_ray * 65536 * n_steps / max(t_fit, 1e-9) / 1e12},
        "inference": {"ms": ms_infer, "tflops": flops_ray * R / (ms_infer / 1e3) / 1e12},
    }


def widened_leg(dev, d, P, cams, cfg, steps=3):
    """The rows around the traced path, timed on the headline workload with
    CUDA events (same traversal configuration, hit cache on): the exact
    adjoint's step (full chain rule, depth/middepth/distortion), the step with
    precomputed per-triangle colours instead of SH, BVH build / refit / save /
    load, and primary rays generated on the device from the cameras.
    `d` holds the workload's device tensors."""
    import torch

    from diff_tritracer import _C

    R = int(d["ro"].shape[0] * d["ro"].shape[1])

    def timed(fn, n=steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    def tracer(**kw):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", **kw)
        if cfg:
            tr.set_traversal(cfg["traversal"], cfg["k"], cfg["stack_depth"])
        tr.build_tri_accel(d["verts"], d["cums"], P, True)
        return tr

    def step_fn(tr, shs, cols):
        def step():
            cache = tr.new_hit_cache(R)
            out = tr.trace_forward(d["ro"], d["rd"], d["verts"], d["sig"], d["npts"], d["cums"], P, shs, 3,
                                   cols if cols is not None else d["empty"], d["opac"], d["scaling"], d["density"],
                                   d["bg"], d["extra"], 1, False, hit_cache=cache).data
            tr.trace_backward(d["ro"], d["rd"], d["bg"], d["verts"], d["sig"], d["npts"], d["cums"], out[0], out[1],
                              P, shs, 3, d["opac"], d["g"], d["go"], d["scaling"], False, colors_precomp=cols,
                              hit_cache=cache)
        return step

    res = {}
    tr = tracer(exact_adjoint=True)
    ms = timed(step_fn(tr, d["shs"], None))
    tr.device_status()
    res["exact_adjoint"] = {"ms_per_step": ms, "mrays": R / ms / 1e3,
                            "step": "refit + forward (depth, middepth, distortion) + exact adjoint, hit cache"}
    del tr
    cols = torch.rand((P, 3), generator=torch.Generator(device=dev).manual_seed(0), device=dev)
    tr = tracer()
    ms = timed(step_fn(tr, d["empty"], cols))
    tr.device_status()
    res["colors_precomp"] = {"ms_per_step": ms, "mrays": R / ms / 1e3,
                             "step": "refit + forward + adjoint with [P, 3] colours instead of SH, hit cache"}
    build_ms = timed(lambda: tr.build_tri_accel(d["verts"], d["cums"], P, True))
    refit_ms = timed(lambda: tr.build_tri_accel(d["verts"], d["cums"], P, False))
    t0 = time.perf_counter()
    blob = tr.save_bvh()
    save_ms = (time.perf_counter() - t0) * 1e3
    other = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    other.load_bvh(blob, d["verts"], d["cums"], P)
    torch.cuda.synchronize()
    load_ms = (time.perf_counter() - t0) * 1e3
    res["bvh"] = {"triangles": P, "build_ms": build_ms, "refit_ms": refit_ms, "save_ms": save_ms,
                  "load_ms": load_ms, "blob_mb": len(blob) / 1e6,
                  "note": "save: device to host blob; load: host blob to device + refit (wall clock, synchronised)"}
    del tr, other
    outs = [(torch.empty((c.H, c.W, 3), device=dev), torch.empty((c.H, c.W, 3), device=dev)) for c in cams]
    gen = _C.OptixTracer()
    ms = timed(lambda: gen.camera_rays(cams, outputs=outs), n=10)
    n_rays = sum(c.H * c.W for c in cams)
    res["camera_rays"] = {"cameras": len(cams), "rays": n_rays, "ms": ms, "mrays": n_rays / ms / 1e3,
                          "bytes_written_gb_s": n_rays * 24 / (ms / 1e3) / 1e9}
    return res


def secondary_leg(dev, steps=3, seed=0, default_only=False):
    """Secondary-ray passes on their benchmark configuration: 500k
    triangles, 20 % dielectric (IOR ~ U[1.3, 1.6]), a 512x1024 lat-long
    environment map (U[0, 1] noise box-filtered 9x9), 2 views of 800x800
    stacked into one [1600, 800] image, up to 2 bounces; forward + adjoint
    through the device ray queue."""
    import torch

    from diff_tritracer import _C, scenes

    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    P = 500_000
    sc = scenes.make_scene(P, seed=seed)
    sec = scenes.secondary_inputs(P, seed=seed)
    cams = scenes.sphere_cameras(2, 800, 800, seed=seed + 3)
    rays = [scenes.camera_rays(c) for c in cams]
    ro = T(np.concatenate([r[0] for r in rays], 0))
    rd = T(np.concatenate([r[1] for r in rays], 0))
    g, go = scenes.upstream_grads(1600, 800, seed=seed)
    g, go = T(g), T(go)
    verts, sig, npts, cums = T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum)
    shs, opac = T(sc.shs), T(sc.opacities)
    mat, ior, env = T(sec["material"]), T(sec["ior"]), T(sec["env"])
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.build_tri_accel(verts, cums, P, True)
    scaling, density = torch.zeros(P, device=dev), torch.zeros(P, device=dev)

    def step():
        color, others, _ = tr.trace_forward_secondary(ro, rd, verts, sig, npts, cums, P, shs, 3, opac, scaling,
                                                      density, mat, ior, env, 2, 2)
        tr.trace_backward_secondary(ro, rd, verts, sig, npts, cums, color, others, P, shs, 3, opac, g, go, mat,
                                    ior, env, 2)

    def timed():
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        tr.reset_stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, tr.stats()

    ms_unsorted = ms_fused = None
    if not default_only:  # the schedule's two parts, each switched off once
        tr.set_sort_secondary(False)
        ms_unsorted, _ = timed()
        tr.set_sort_secondary(True)
        tr.set_split_forward(False)
        ms_fused, _ = timed()
        tr.set_split_forward(True)
    ms, st = timed()
    tr.device_status()
    R = 1600 * 800
    return {"workload": "500k triangles, 20% dielectric, env 512x1024, 2 views 800x800, 2 bounces",
            "pixels_per_step": R, "rays_per_step": st["rays"] / steps, "ms_per_step": ms,
            "primary_mrays": R / ms / 1e3, "all_rays_mrays": st["rays"] / steps / ms / 1e3,
            "ms_per_step_spawn_order": ms_unsorted, "ms_per_step_without_split": ms_fused,
            "step": "forward (3 trace levels, spawned levels sorted by direction and origin and traced "
                    "as a traversal-only pass plus a shading pass, + 3 resolves) + adjoint (all levels, one launch)"}


def views_leg(dev, name, steps, warmup=3, no_autotune=False, world=1, local=0, sample_clocks=False):
    """Batched uneven views: every step is one CUDA-graph replay of refit +
    forward + adjoint over all 16 views (ViewBatch), after autotuning.
    Returns the timed figures (the caller reports them)."""
    import torch
    import torch.distributed as dist

    from diff_tritracer import _C
    from diff_tritracer.autotune import autotune
    from diff_tritracer.batch import ViewBatch

    P = WORKLOADS[name][0]
    sc, rays_np, ups_np = make_workload(name)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    scene = dict(triangles_points=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), num_points_per_triangle=T(sc.num_points),
                 cumsum_of_points_per_triangle=T(sc.cumsum), number_of_points=P, shs=T(sc.shs),
                 opacities=T(sc.opacities), scaling=torch.zeros(P, device=dev), density_factor=torch.zeros(P, device=dev))
    shapes = [r[0].shape[:2] for r in rays_np]
    R = int(sum(h * w for h, w in shapes))
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    bg = torch.zeros(3, device=dev)
    eager = ViewBatch(tr, shapes, scene, 3, bg, graph=False)
    eager.set_rays([(T(a), T(b)) for a, b in rays_np])
    eager.set_upstream([(T(a), T(b)) for a, b in ups_np])
    tuned = None if no_autotune else autotune(tr, eager.step, key=name, iters=2, prepare=eager.fit_hit_cache)
    # kernels per step, counted on an eager step (graph replays are not seen by the host counter)
    eager.fit_hit_cache()
    tr.reset_stats()
    eager.step()
    per_step = tr.stats()["kernel_launches"]
    del eager
    vb = ViewBatch(tr, shapes, scene, 3, bg, graph=True)
    vb.set_rays([(T(a), T(b)) for a, b in rays_np])
    vb.set_upstream([(T(a), T(b)) for a, b in ups_np])
    cache_use = vb.fit_hit_cache()
    for _ in range(max(3, warmup)):
        vb.step()
    torch.cuda.synchronize()
    tr.device_status()
    sampler = ClockSampler(local) if sample_clocks else None
    tr.reset_stats()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        vb.step()
    t1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    ms = t0.elapsed_time(t1)
    st = tr.stats()
    tr.device_status()
    ms = slowest_rank_ms(ms, world, dev)
    return {
        "value": world * R * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps, "steps": steps,
        "gpu_launches": int(per_step * steps), "clocks": clocks,
        "config": {"workload": name, "triangles": P, "views": len(shapes),
                   "resolutions": [f"{h}x{w}" for h, w in shapes], "rays_per_step": R,
                   "step": "one CUDA-graph replay: refit + forward + adjoint over all views",
                   "traversal": ({k: tuned.get(k) for k in ("traversal", "k", "stack_depth", "split", "collect")} if tuned else "default"),
                   "autotune_ms": tuned.get("all") if tuned else None,
                   "hit_cache": {"pool_queries": cache_use["pool_cap"], "later_queries": cache_use["pool_used"],
                                 "replays_per_ray": st["hit_cache_replays"] / max(st["rays"], 1),
                                 "queries_per_ray": st["queries"] / max(st["rays"], 1)},
                   "hits_per_ray": {"evaluated": st["evaluated_hits"] / max(st["rays"], 1),
                                    "blended": st["blended_hits"] / max(st["rays"], 1)}},
    }


def run_views(args, world, rank, local, dev):
    """The batched workload as the bench's main line."""
    import torch.distributed as dist

    r = views_leg(dev, args.workload, args.steps, args.warmup, args.no_autotune, world, local, sample_clocks=True)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": r["value"], "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": r["config"],
        "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
    }), flush=True)


def c1_leg(dev, steps=50):
    """The small plain-method configuration (100k triangles, one 400x400
    view): refit + forward + adjoint per step, hit cache on, CUDA events."""
    import torch

    from diff_tritracer import _C

    sc, ro_np, rd_np, g_np, go_np = make_workload("c1_100k_1x400")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ro, rd, g, go = T(ro_np), T(rd_np), T(g_np), T(go_np)
    verts, sig, npts, cums = T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum)
    shs, opac = T(sc.shs), T(sc.opacities)
    P = sc.P
    z = lambda: torch.zeros(P, device=dev)
    bg, extra, empty, scaling, density = torch.zeros(3, device=dev), torch.zeros(5, device=dev), \
        torch.empty(0, device=dev), z(), z()
    R = ro.shape[0] * ro.shape[1]
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.build_tri_accel(verts, cums, P, True)

    def step():
        cache = tr.new_hit_cache(R)
        out = tr.trace_forward(ro, rd, verts, sig, npts, cums, P, shs, 3, empty, opac, scaling, density, bg, extra,
                               1, False, hit_cache=cache).data
        tr.trace_backward(ro, rd, bg, verts, sig, npts, cums, out[0], out[1], P, shs, 3, opac, g, go, scaling, False,
                          hit_cache=cache)

    for _ in range(5):
        step()
    torch.cuda.synchronize()
    tr.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    st = tr.stats()
    tr.device_status()
    return {"workload": "c1_100k_1x400", "rays_per_step": R, "ms_per_step": ms, "mrays": R / ms / 1e3,
            "step": "refit + forward + adjoint, hit cache on, default traversal",
            "hits_per_ray": {"evaluated": st["evaluated_hits"] / max(st["rays"], 1),
                             "blended": st["blended_hits"] / max(st["rays"], 1)}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_1M_4x800", choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=20,
                    help="steps of the end-to-end leg (the same count as the device-timed steps by default)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ref-budget", type=float, default=3.0, help="seconds of CPU work per reference step")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default traversal configuration")
    ap.add_argument("--no-proposal", action="store_true", help="skip the learned-proposal leg")
    ap.add_argument("--proposal-small", action="store_true", help="learned-proposal leg at profiling size")
    ap.add_argument("--no-secondary", action="store_true", help="skip the secondary-ray leg")
    ap.add_argument("--secondary-only", action="store_true",
                    help="run only the secondary-ray leg, in its default schedule, for --steps steps (profiling)")
    ap.add_argument("--no-widened", action="store_true",
                    help="skip the leg timing the exact adjoint, precomputed colours, BVH files and camera rays")
    ap.add_argument("--no-c4", action="store_true", help="skip the batched 3M-triangle, 16-view leg")
    ap.add_argument("--no-c1", action="store_true", help="skip the 100k-triangle, one-view leg")
    ap.add_argument("--no-hit-cache", action="store_true",
                    help="adjoint re-traverses every query instead of replaying the forward's")
    ap.add_argument("--split-forward", action="store_true",
                    help="run the plain forward as a traversal-only pass plus a shading pass")
    ap.add_argument("--collect-queries", type=int, default=None,
                    help="split forward: queries per ray the traversal-only pass stores (0 = all)")
    ap.add_argument("--traversal", default=None, choices=["packets16", "packets32", "lanes32", "lanes24"],
                    help="fix the traversal configuration instead of autotuning it")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    import diff_tritracer
    from diff_tritracer import _C
    from diff_tritracer.autotune import autotune

    if args.secondary_only:
        print(json.dumps({"secondary": secondary_leg(dev, steps=args.steps, default_only=True)}), flush=True)
        return

    name = args.workload
    if name.startswith("c4"):
        return run_views(args, world, rank, local, dev)
    P, views, H, W = WORKLOADS[name]
    sc, ro_np, rd_np, g_np, go_np = make_workload(name)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ro, rd, g, go = T(ro_np), T(rd_np), T(g_np), T(go_np)
    verts, sig, npts, cums = T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum)
    shs, opac = T(sc.shs), T(sc.opacities)
    bg = torch.zeros(3, device=dev)
    extra = torch.zeros(5, device=dev)
    scaling = torch.zeros(P, device=dev)
    density = torch.zeros(P, device=dev)
    empty = torch.empty(0, device=dev)
    HH, WW = ro.shape[0], ro.shape[1]
    R = HH * WW

    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    tr.build_tri_accel(verts, cums, P, True)
    tr.set_split_forward(args.split_forward)
    if args.collect_queries is not None:
        tr.set_collect_queries(args.collect_queries)
    use_cache = not args.no_hit_cache

    def step(cached=use_cache):
        # the hit cache is the step's activation: allocated (caching allocator) and filled every step
        cache = tr.new_hit_cache(R) if cached else None
        out = tr.trace_forward(ro, rd, verts, sig, npts, cums, P, shs, 3, empty, opac, scaling, density, bg, extra,
                               1, False, hit_cache=cache).data
        tr.trace_backward(ro, rd, bg, verts, sig, npts, cums, out[0], out[1], P, shs, 3, opac, g, go, scaling, False,
                          hit_cache=cache)

    # kernel-level timing: forward and adjoint each bracketed by events
    def timed_kernels(n, cached=use_cache):
        fwd_ms, bwd_ms = [], []
        for _ in range(n):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            tr.build_tri_accel(verts, cums, P, False)
            cache = tr.new_hit_cache(R) if cached else None
            e[0].record()
            out = tr.trace_forward(ro, rd, verts, sig, npts, cums, P, shs, 3, empty, opac, scaling, density, bg,
                                   extra, 2, False, hit_cache=cache).data
            e[1].record()
            tr.trace_backward(ro, rd, bg, verts, sig, npts, cums, out[0], out[1], P, shs, 3, opac, g, go, scaling,
                              False, hit_cache=cache)
            e[2].record()
            torch.cuda.synchronize()
            fwd_ms.append(e[0].elapsed_time(e[1]))
            bwd_ms.append(e[1].elapsed_time(e[2]))
        return float(np.mean(fwd_ms)), float(np.mean(bwd_ms))

    tuned = None
    if args.traversal:
        mode, num = args.traversal.rstrip("0123456789"), int(args.traversal.lstrip("acdeklnpst"))
        tr.set_traversal(mode, k=num if mode == "packets" else 16, stack_depth=num if mode == "lanes" else 32)
        tuned = {"traversal": mode, "k": num if mode == "packets" else 16,
                 "stack_depth": num if mode == "lanes" else 32}
    elif not args.no_autotune:
        tuned = autotune(tr, step, key=f"{name}", iters=2)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    tr.device_status()

    # ---------------- timed region: exactly K steps
    sampler = ClockSampler(local)
    tr.reset_stats()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        step()
    t1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    elapsed_ms = t0.elapsed_time(t1)
    st = tr.stats()
    tr.device_status()
    elapsed_ms = slowest_rank_ms(elapsed_ms, world, dev)
    ms_per_step = elapsed_ms / args.steps
    value = world * R * args.steps / (elapsed_ms / 1e3) / 1e6

    # the same timed protocol with the adjoint re-traversing every query
    value_retrace = None
    if use_cache:
        for _ in range(2):
            step(False)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0.record()
        for _ in range(args.steps):
            step(False)
        t1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        value_retrace = world * R * args.steps / (slowest_rank_ms(t0.elapsed_time(t1), world, dev) / 1e3) / 1e6

    # traversal work of one step, counted outside the timed region (the
    # counters cost the traversal a few per cent, so they are off while timing)
    tr.set_work_counters(True)
    tr.reset_stats()
    step()
    st_work = tr.stats()
    tr.set_work_counters(False)

    # ---------------- roofline of the dominant kernel (adjoint)
    fwd_ms, bwd_ms = timed_kernels(3)
    fwd_plain_ms, bwd_retrace_ms = timed_kernels(2, cached=False) if use_cache else (fwd_ms, bwd_ms)
    # the forward under each schedule, and the device time of its two passes
    # (debug events around the traversal-only pass and the shading pass)
    schedules = {}
    if use_cache:
        cur = (tuned or {}).get("split", args.split_forward), (tuned or {}).get("collect", args.collect_queries or 1)
        for sname, split, collect in (("fused", False, 1), ("split_first", True, 1), ("split_two", True, 2),
                                      ("split_all", True, 0)):
            tr.set_split_forward(split)
            tr.set_collect_queries(collect)
            step()  # first launches of this schedule's kernels, untimed
            f_ms = timed_kernels(3)[0]
            passes = []
            for _ in range(3):
                cache = tr.new_hit_cache(R)
                tr.trace_forward(ro, rd, verts, sig, npts, cums, P, shs, 3, empty, opac, scaling, density, bg, extra,
                                 2, True, hit_cache=cache)
                passes.append(tr.forward_pass_times())
            schedules[sname] = {"forward_ms": f_ms, "collect_ms": float(np.mean([x[0] for x in passes])),
                                "shade_ms": float(np.mean([x[1] for x in passes]))}
        tr.set_split_forward(bool(cur[0]))
        tr.set_collect_queries(int(cur[1]))
    rays_step = st["rays"] / args.steps
    evals = st["evaluated_hits"] / args.steps
    blends = st["blended_hits"] / args.steps
    k_cache = int(tuned["k"]) if tuned else 16
    packets = (tuned or {}).get("traversal", "packets") == "packets"
    fwd_b, bwd_b = algorithmic_bytes(rays_step, evals, blends, cache_k=k_cache if use_cache else 0,
                                     colors=packets)
    peak, peak_kind = peaks()
    dominant = "adjoint" if bwd_ms >= fwd_ms else "forward"
    dom_bytes, dom_ms = (bwd_b, bwd_ms) if dominant == "adjoint" else (fwd_b, fwd_ms)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"traffic_{name}.txt")
    if os.path.exists(tfile):
        for ln in open(tfile):
            parts = ln.split()
            if len(parts) == 2 and parts[0] == dominant:
                traffic = float(parts[1])

    # ---------------- end to end through the public API (host buffers)
    tracer_mod = diff_tritracer.Tracer("forward.ptx", "backward.ptx", hit_cache=use_cache)
    tracer_mod.tracer = tr
    tr.use_hit_cache = use_cache
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    ro_h, rd_h, g_h = pin(ro_np), pin(rd_np), pin(g_np)
    color_h = torch.empty((3, HH, WW), dtype=torch.float32).pin_memory()
    verts_p = verts.clone().requires_grad_(True)
    sig_p, opac_p, shs_p = sig.clone().requires_grad_(True), opac.clone().requires_grad_(True), \
        shs.clone().requires_grad_(True)
    settings = diff_tritracer.TracerSettings(bg=bg, scale_modifier=1.0, sh_degree=3, debug=False, rebuild_gas=1,
                                             extra_params=extra)

    copy_stream = torch.cuda.Stream(dev)
    # double-buffered rays: each step's rays are uploaded on the copy stream
    # during the previous step, as a training loop's data loader would
    ray_bufs = [(torch.empty(ro_h.shape, device=dev), torch.empty(rd_h.shape, device=dev)) for _ in range(2)]
    ray_ready = [torch.cuda.Event(), torch.cuda.Event()]

    def upload_rays(slot):
        with torch.cuda.stream(copy_stream):
            ray_bufs[slot][0].copy_(ro_h, non_blocking=True)
            ray_bufs[slot][1].copy_(rd_h, non_blocking=True)
            ray_ready[slot].record(copy_stream)

    def e2e_step(i):
        # the upstream gradient comes in on the copy stream while the forward
        # runs; the image goes out, and the next step's rays come in, while the
        # adjoint runs; the step ends when all three have
        main = torch.cuda.current_stream(dev)
        slot = i % 2
        main.wait_event(ray_ready[slot])
        ro_d, rd_d = ray_bufs[slot]
        with torch.cuda.stream(copy_stream):
            g_d = g_h.to(dev, non_blocking=True)
            g_ready = torch.cuda.Event()
            g_ready.record(copy_stream)
        g_d.record_stream(main)
        color, _, _, _, _, _ = tracer_mod(ro_d, rd_d, verts_p, sig_p, npts, cums, P, opac_p, scaling, density,
                                          shs_p, None, settings)
        fwd_done = torch.cuda.Event()
        fwd_done.record(main)
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(fwd_done)  # the other slot's last reader (the previous step) is done
            color_h.copy_(color.detach(), non_blocking=True)
        color.record_stream(copy_stream)
        upload_rays(1 - slot)
        main.wait_event(g_ready)
        color.backward(g_d)
        main.wait_stream(copy_stream)

    def link_gbs():
        # pinned host <-> device bandwidth as this run sees it (the machine is
        # shared: other jobs' traffic shows here and in the e2e number alike)
        out = []
        for src, dst in ((ro_h, ray_bufs[0][0]), (color, color_h)):
            with torch.cuda.stream(copy_stream):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(copy_stream)
                for _ in range(3):
                    dst.copy_(src, non_blocking=True)
                b.record(copy_stream)
            torch.cuda.synchronize()
            out.append(3 * src.numel() * 4 / (a.elapsed_time(b) / 1e3) / 1e9)
        return out

    color = torch.empty((3, HH, WW), device=dev)
    link_before = link_gbs()
    upload_rays(0)
    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.e2e_steps + 1)]
    ev[0].record()
    for i in range(args.e2e_steps):  # each timed step uploads one step's rays, gradient and image
        e2e_step(2 + i)
        ev[i + 1].record()
    torch.cuda.synchronize()
    e2e_ms = ev[0].elapsed_time(ev[-1])
    e2e_step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.e2e_steps)]
    e2e_ms = slowest_rank_ms(e2e_ms, world, dev)
    e2e_value = world * R * args.e2e_steps / (e2e_ms / 1e3) / 1e6
    h2d = ro_h.numel() * 4 + rd_h.numel() * 4 + g_h.numel() * 4
    d2h = color_h.numel() * 4
    link_after = link_gbs()

    # ---------------- CPU baseline (rank 0, N = 1)
    prop = None
    if rank == 0 and world == 1 and not args.no_proposal:
        prop = proposal_leg(dev, small=args.proposal_small)
    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        secondary = secondary_leg(dev)
    widened = None
    if rank == 0 and world == 1 and not args.no_widened:
        from diff_tritracer import scenes

        tensors = dict(verts=verts, sig=sig, npts=npts, cums=cums, shs=shs, opac=opac, ro=ro, rd=rd, g=g, go=go,
                       bg=bg, extra=extra, empty=empty, scaling=scaling, density=density)
        widened = widened_leg(dev, tensors, P, scenes.sphere_cameras(views, H, W, seed=0), tuned)

    c4 = c1 = None
    if rank == 0 and world == 1 and not args.no_c4:
        r = views_leg(dev, "c4_3M_16views", steps=5)
        c4 = {"value_mrays": r["value"], "ms_per_step": r["ms_per_step"], "steps": r["steps"], **r["config"]}
    if rank == 0 and world == 1 and not args.no_c1:
        c1 = c1_leg(dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(name, sc, ro_np, rd_np, g_np, go_np)[0]

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    launches_per_step = st["kernel_launches"] / args.steps
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "triangles": P, "views": views, "H": H, "W": W, "rays_per_step": R,
                   "step": "BVH refit + forward trace + adjoint trace",
                   "hit_cache": ({"on": "the forward stores its k-closest queries (the step's activation: "
                                        "(k+1)*8 B/ray for first queries + a pool for later ones); the adjoint "
                                        "replays them instead of re-traversing",
                                  "value_with_retracing_adjoint": value_retrace}
                                 if use_cache else "off: the adjoint re-traverses every query"),
                   "l2": "inputs larger than L2 (scene + BVH + rays ~0.5 GB per step)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "traversal": ({k: tuned.get(k) for k in ("traversal", "k", "stack_depth", "split", "collect")} if tuned else "default"),
                   "hits_per_ray": {"evaluated": evals / max(rays_step, 1), "blended": blends / max(rays_step, 1)},
                   "traversal_per_ray": {k: st_work[k] / max(st_work["rays"], 1)
                                         for k in ("queries", "node_visits", "triangle_tests",
                                                   "packet_node_visits")}},
        "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "diff_tritracer.Tracer autograd forward+backward, pinned host rays/grads in, image out "
                        "(on a copy stream: gradient upload under the forward; image download and the next "
                        "step's ray upload, double-buffered, under the adjoint)",
                "step_ms": e2e_step_ms,
                "link_gbs": {"h2d_before": link_before[0], "d2h_before": link_before[1], "h2d_after": link_after[0],
                             "d2h_after": link_after[1],
                             "note": "pinned copies of one step's rays / image timed alone before and after the "
                                     "e2e steps (the host link is shared with other jobs)"}},
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "roofline": {"bound": "hbm", "kernel": dominant + (" (traversal-only pass + shading pass)"
                                                          if dominant == "forward" and (tuned or {}).get("split")
                                                          else ""), "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms,
                     "forward_ms": fwd_ms, "adjoint_ms": bwd_ms,
                     "forward_without_cache_ms": fwd_plain_ms, "adjoint_retrace_ms": bwd_retrace_ms,
                     "forward_by_schedule": schedules,
                     "forward_frac": fwd_b / (fwd_ms / 1e3) / 1e9 / peak},
        "cpu_baseline": cpu,
        "proposal": prop,
        "secondary": secondary,
        "widened": widened,
        "c4": c4,
        "c1": c1,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
