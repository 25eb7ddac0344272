"""Shared helpers of the GPU parity tests: run the package's CUDA path and the
FP64 oracle on the same seeded inputs."""
from __future__ import annotations

import numpy as np
import torch

import diff_tritracer
from diff_tritracer import scenes

DEV = torch.device("cuda:0")

# A ray whose decisions (alpha vs 1/255, T(1-alpha) vs 1e-4) sit within this
# relative distance of a threshold in the FP64 oracle may legitimately go the
# other way in FP32; such rays are excluded from the per-pixel comparisons.
MARGIN = 1e-5


def T(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return t if dtype is None else t.to(dtype)


def settings(bg=None, sh_degree=3, rebuild=0, extra=None, debug=False):
    bg = torch.zeros(3, device=DEV) if bg is None else T(np.asarray(bg, np.float32))
    ex = torch.zeros(5, device=DEV) if extra is None else T(np.asarray(extra, np.float32))
    return diff_tritracer.TracerSettings(bg=bg, scale_modifier=1.0, sh_degree=sh_degree, debug=debug,
                                         rebuild_gas=rebuild, extra_params=ex)


def gpu_forward(tracer, sc, ro, rd, st, scaling=None, density=None):
    """Direct _C call (no autograd): returns numpy color, others, scaling, density, max_blending."""
    P = sc.P
    scaling = torch.zeros(P, device=DEV) if scaling is None else T(scaling)
    density = torch.zeros(P, device=DEV) if density is None else T(density)
    res = tracer.trace_forward(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), P,
                               T(sc.shs), st.sh_degree, torch.empty(0, device=DEV), T(sc.opacities), scaling, density,
                               st.bg, st.extra_params, st.rebuild_gas, st.debug)
    color, others, gpu_time, scaling, density, maxb = res.data
    torch.cuda.synchronize()
    return {k: v.detach().cpu().numpy() for k, v in dict(color=color, others=others, scaling=scaling,
                                                         density=density, max_blending=maxb,
                                                         gpu_time=gpu_time).items()}


def gpu_backward(tracer, sc, ro, rd, st, colors, others, g, go):
    res = tracer.trace_backward(T(ro), T(rd), st.bg, T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points),
                                T(sc.cumsum), T(colors), T(others), sc.P, T(sc.shs), st.sh_degree, T(sc.opacities),
                                T(g), T(go), torch.zeros(sc.P, device=DEV), st.debug)
    dtri, dsig, dop, dsh = res.data
    torch.cuda.synchronize()
    return dict(dtri=dtri.cpu().numpy(), dsigma=dsig.cpu().numpy().reshape(-1), dopac=dop.cpu().numpy().reshape(-1),
                dsh=dsh.cpu().numpy())


def rel_norm(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def flagged_prims(rec, H, W, ok_mask):
    """Primitives visited by any excluded ray (from the oracle's record)."""
    bad = ~ok_mask.reshape(-1)
    ids = rec.rec_ids[bad]
    return np.unique(ids[ids >= 0])
