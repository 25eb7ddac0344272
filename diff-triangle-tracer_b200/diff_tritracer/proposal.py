"""Learned proposal: a small ray MLP that predicts, per ray, the interval
[t_near, t_far] holding the hits the tracer's march visits, so the traversal
can be clipped to it (tt_view.interval). No counterpart in the reference,
which traces every ray from the camera to the far plane.

The network, its training step (forward, loss, backward, weight gradients)
and its inference run in the library's tensor-core kernels (tt_mlp_*); this
module owns the parameter tensors and drives data collection, training,
validation of the margins and the clipped trace.

The network sees each ray's line only: the origin is moved along the ray
to its closest approach to the scene centre (o' = o + s d) and the outputs
are t - s, so rays of cameras it never saw look like its training rays.

Training targets come from the plain tracer itself: a forward with hit
records gives each ray's first visited hit t_first, its last visited hit
t_last and whether it terminated on the transmittance cut-off. Targets:
t_near = t_first (-1 for a ray without hits: no t_near term), t_far = t_last
for a terminated ray, else s + `far_target` (no far clip: the ray runs to the
end of the scene anyway). A t_near above its target would cut hits off and
change the image, so it weighs `near_weight` times more; a t_far below its
target only costs a continuation and weighs `far_weight`.

At trace time an interval is [t_near - margin_near, t_far + margin_far], with
t_far = +inf when t_far + margin_far - s reaches `far_cap`. A ray whose
interval is too short at the far end continues beyond it and one with no hit
inside is traced again (both exact); only a t_near beyond the ray's first
hits changes the result. On triangle clouds the first hit of a ray is too
erratic to predict within a safe margin, so the default margin_near switches
the near clip off and the far clip carries the gain.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

PARAMS = _lib.TT_MLP_PARAMS
NO_NEAR_CLIP = 1.0e4  # a margin_near that puts every t_near before the ray origin
PARTIAL = _lib.TT_MLP_PARTIAL
IN, HID, OUT_ROWS = 80, 64, 16
ROWS = (HID, HID, HID, OUT_ROWS)
OFF = (0, HID * IN, 2 * HID * IN, 3 * HID * IN)


def init_params(seed=0):
    """He-uniform weights on the real inputs, zero biases, zero for every
    weight fed by the zero input and for the unused output rows."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    fan = (78, HID, HID, HID)
    for l in range(4):
        w = np.zeros((ROWS[l], IN), np.float32)
        rows = 2 if l == 3 else ROWS[l]
        b = math.sqrt(6.0 / fan[l]) * (0.1 if l == 3 else 1.0)
        w[:rows, :fan[l]] = rng.uniform(-b, b, (rows, fan[l]))
        p[OFF[l]:OFF[l] + ROWS[l] * IN] = w.reshape(-1)
    return p


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Proposal:
    """Parameters, Adam state and scratch of the proposal network on one
    device, driven through the tracer handle `tracer` (an OptixTracer, for
    its error reporting and status word)."""

    def __init__(self, tracer, origin_scale=1.0 / 3.0, t_shift=0.0, t_scale=1.0, center=(0.0, 0.0, 0.0), seed=0):
        self.tracer = tracer
        dev = tracer.device
        self.device = dev
        self.master = torch.from_numpy(init_params(seed)).to(dev)
        self.adam_m = torch.zeros(PARAMS, dtype=torch.float32, device=dev)
        self.adam_v = torch.zeros(PARAMS, dtype=torch.float32, device=dev)
        self.weights = torch.zeros(PARAMS, dtype=torch.int16, device=dev)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        self.partial = torch.zeros((sms, PARTIAL), dtype=torch.float32, device=dev)
        self.origin_scale, self.t_shift, self.t_scale = float(origin_scale), float(t_shift), float(t_scale)
        self.center = tuple(float(c) for c in center)
        self.steps = 0
        self.far_target = 3.0   # t - s of "no far clip"
        self.far_cap = 2.5      # t_far - s beyond which no far clip is applied
        self.margin_near = NO_NEAR_CLIP
        self.margin_far = 0.05
        self.update()

    # -------------------------------------------------------------- C ABI
    def _net(self):
        n = _lib.TtMlp()
        n.weights, n.master = _ptr(self.weights), _ptr(self.master)
        n.adam_m, n.adam_v, n.partial = _ptr(self.adam_m), _ptr(self.adam_v), _ptr(self.partial)
        n.partial_ctas = int(self.partial.shape[0])
        n.origin_scale, n.t_shift, n.t_scale = self.origin_scale, self.t_shift, self.t_scale
        n.center[0], n.center[1], n.center[2] = self.center
        return n

    def update(self):
        """Refreshes the BF16 tensor-core copy from the FP32 master weights."""
        n = self._net()
        check(self.tracer._h, lib.tt_mlp_update(self.tracer._h, ctypes.byref(n), _stream()))

    def train_step(self, rays, targets, lr=1e-3, near_weight=8.0, far_weight=3.0, betas=(0.9, 0.999), eps=1e-8,
                   loss_out=None):
        """One Adam step on a batch: rays [n, 6] (origin, direction), targets
        [n, 2] (t_near, t_far), float32 device tensors. Writes the batch's mean
        loss into loss_out (a 1-element device tensor) when given."""
        rays = rays.contiguous()
        targets = targets.contiguous()
        n = int(rays.shape[0])
        self.steps += 1
        st = _lib.TtMlpStep(float(lr), float(betas[0]), float(betas[1]), float(eps), self.steps, float(near_weight),
                            float(far_weight))
        net = self._net()
        lp = _ptr(loss_out) if loss_out is not None else ctypes.c_void_p(0)
        check(self.tracer._h, lib.tt_mlp_train_step(self.tracer._h, ctypes.byref(net), ctypes.byref(st), _ptr(rays),
                                                    _ptr(targets), n, lp, _stream()))
        self._keep = (rays, targets)

    def predict(self, rays):
        """Raw (t_near, t_far) for rays [n, 6] -> [n, 2]."""
        rays = rays.contiguous()
        out = torch.empty((rays.shape[0], 2), dtype=torch.float32, device=self.device)
        net = self._net()
        check(self.tracer._h, lib.tt_mlp_predict(self.tracer._h, ctypes.byref(net), _ptr(rays), int(rays.shape[0]),
                                                 _ptr(out), _stream()))
        self._keep = (rays,)
        return out

    def intervals(self, rays, margin_near=None, margin_far=None, far_cap=None, out=None):
        """Clip intervals [2, H, W] for views given as (ray_o, ray_d) pairs."""
        mn = self.margin_near if margin_near is None else margin_near
        mf = self.margin_far if margin_far is None else margin_far
        cap = self.far_cap if far_cap is None else far_cap
        vs = (_lib.TtView * len(rays))()
        outs = []
        keep = []
        for i, (ro, rd) in enumerate(rays):
            H, W = int(ro.shape[0]), int(ro.shape[1])
            ro, rd = ro.contiguous(), rd.contiguous()
            vs[i].H, vs[i].W = H, W
            vs[i].ray_o, vs[i].ray_d = _ptr(ro), _ptr(rd)
            iv = out[i] if out is not None else torch.empty((2, H, W), dtype=torch.float32, device=self.device)
            outs.append(iv)
            keep += [ro, rd]
        ptrs = (ctypes.c_void_p * len(rays))(*[iv.data_ptr() for iv in outs])
        net = self._net()
        check(self.tracer._h, lib.tt_mlp_intervals(self.tracer._h, ctypes.byref(net), vs, len(rays), ptrs,
                                                   float(mn), float(mf), float(cap), _stream()))
        self._keep = tuple(keep)
        return outs

    # -------------------------------------------------------------- state
    def state_dict(self):
        return {"master": self.master.clone(), "origin_scale": self.origin_scale, "t_shift": self.t_shift,
                "t_scale": self.t_scale, "center": self.center, "far_target": self.far_target,
                "far_cap": self.far_cap, "margin_near": self.margin_near, "margin_far": self.margin_far}

    def load_state_dict(self, d):
        self.master.copy_(d["master"].to(self.device))
        for k in ("origin_scale", "t_shift", "t_scale", "far_target", "far_cap", "margin_near", "margin_far"):
            setattr(self, k, float(d[k]))
        self.center = tuple(float(c) for c in d["center"])
        self.update()

    def offsets(self, rays):
        """s per ray [n, 6]: distance from the origin to the closest approach."""
        o = rays[:, :3] - torch.tensor(self.center, device=rays.device)
        d = rays[:, 3:6]
        return -(o * d).sum(1) / (d * d).sum(1)


# ------------------------------------------------------------------ data
def targets_from_record(rec, s, far_target):
    """Training targets [n, 2] from hit records [3, n] (t_first, t_last,
    terminated) of the plain tracer; s [n] are the rays' closest-approach
    offsets and far_target the t - s of "no far clip"."""
    t_first, t_last, term = rec[0], rec[1], rec[2]
    hit = torch.isfinite(t_first)
    near = torch.where(hit, t_first, torch.full_like(t_first, -1.0))
    far = torch.where(hit & (term > 0.5), t_last, s + far_target)
    return torch.stack([near, far], 1)


def collect(prop, tracer, scene, views, far_target=None, bg=None):
    """Traces `views` (list of (ray_o, ray_d) [H, W, 3]) with the plain
    tracer and returns (rays [N, 6], targets [N, 2], far_target). `scene` is
    a dict of device tensors: verts, sigma, npts, cums, shs, opac, P. Without
    a far_target, 0.5 beyond the last hit seen (relative to s) is used."""
    dev = tracer.device
    bg = torch.zeros(3, device=dev) if bg is None else bg
    rays, recs = [], []
    for i in range(0, len(views), 32):
        chunk = views[i:i + 32]
        records = [torch.empty((3, ro.shape[0], ro.shape[1]), dtype=torch.float32, device=dev) for ro, _ in chunk]
        scaling = torch.zeros(scene["P"], device=dev)
        dens = torch.zeros(scene["P"], device=dev)
        tracer.trace_forward_views(chunk, scene["verts"], scene["sigma"], scene["npts"], scene["cums"], scene["P"],
                                   scene["shs"], 3, scene["opac"], scaling, dens, bg, 2, records=records)
        for (ro, rd), rec in zip(chunk, records):
            rays.append(torch.cat([ro.reshape(-1, 3), rd.reshape(-1, 3)], 1))
            recs.append(rec.reshape(3, -1))
    rays = torch.cat(rays, 0).contiguous()
    rec = torch.cat(recs, 1)
    s = prop.offsets(rays)
    if far_target is None:
        hit = torch.isfinite(rec[1])
        far_target = float((rec[1] - s)[hit].max().item()) + 0.5 if bool(hit.any()) else 3.0
    return rays, targets_from_record(rec, s, far_target).contiguous(), far_target


def fit(prop, rays, targets, epochs=20, batch=65536, lr=1e-3, near_weight=8.0, far_weight=3.0, seed=0,
        lr_final=None):
    """Adam over shuffled batches; returns the per-step losses (one sync at
    the end). The learning rate decays cosine-wise to lr_final (default
    lr / 10)."""
    dev = prop.device
    n = int(rays.shape[0])
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    losses = torch.zeros(total, dtype=torch.float32, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lr_final = lr * 0.1 if lr_final is None else lr_final
    k = 0
    for _ in range(epochs):
        perm = torch.randperm(n, device=dev, generator=g)
        r, t = rays[perm].contiguous(), targets[perm].contiguous()
        for s in range(steps_per_epoch):
            cur = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * k / max(1, total - 1)))
            prop.train_step(r[s * batch:(s + 1) * batch], t[s * batch:(s + 1) * batch], lr=cur,
                            near_weight=near_weight, far_weight=far_weight, loss_out=losses[k:k + 1])
            k += 1
    return losses.cpu().numpy()


def interval_stats(prop, rays, targets, margin_near=None, margin_far=None, far_cap=None):
    """How intervals [t_near - m_n, t_far + m_f] of `prop` fit the targets:
    near misses (t_near beyond the first hit: hits skipped, among rays with
    hits), far misses (a terminated ray's last hit beyond a finite t_far: a
    continuation, among terminated rays), false far clips (a ray that does not
    terminate given a finite t_far: a continuation, among those rays) and the
    share of terminated rays whose t_far is finite."""
    mn = prop.margin_near if margin_near is None else margin_near
    mf = prop.margin_far if margin_far is None else margin_far
    cap = prop.far_cap if far_cap is None else far_cap
    pred = prop.predict(rays)
    s = prop.offsets(rays)
    tn = pred[:, 0] - mn
    clip = (pred[:, 1] - s + mf) < cap
    hit = targets[:, 0] >= 0
    term = (targets[:, 1] - s) < prop.far_target - 1e-3
    f = lambda x: float(x.float().mean().item()) if x.numel() else 0.0
    return {"near_miss": f((tn > targets[:, 0])[hit]),
            "far_miss": f((clip & (pred[:, 1] + mf < targets[:, 1]))[term]),
            "false_far_clip": f(clip[~term]),
            "far_clipped": f(clip[term]),
            "far_err_median": float((pred[:, 1] - targets[:, 1])[term].abs().median().item()) if bool(term.any())
            else 0.0,
            "terminated": f(term)}
