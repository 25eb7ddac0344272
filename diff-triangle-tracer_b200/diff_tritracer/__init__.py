"""diff_tritracer: differentiable k-closest-hit triangle tracer for NVIDIA B200.

Same Python surface as the reference package (diff_tritracer/__init__.py:37-283
there): ``TracerSettings``, ``Tracer(forward_ptx, backward_ptx)`` whose
``forward`` takes the same 13 arguments and returns
``(color, gpu_time, scaling, density_factor, others, max_blending)``, and an
autograd function whose backward yields gradients for the triangle vertices,
sigma, SH coefficients and opacities. The compute runs in hand-written sm_100a
kernels behind the C ABI of libtritracer.so (include/tritracer.h); there is no
CPU path.
"""

from __future__ import annotations

from typing import NamedTuple

import torch
import torch.nn as nn

from . import _C

__all__ = ["TracerSettings", "Tracer", "_C"]


class TracerSettings(NamedTuple):
    bg: torch.Tensor
    scale_modifier: float  # accepted, unused (as in the reference)
    sh_degree: int
    debug: bool
    rebuild_gas: int  # 0 rebuild the BVH, 1 refit it, 2 keep it
    extra_params: torch.Tensor  # variant parameters [r, cx, cy, cz, samples]


def cpu_deep_copy_tuple(values):
    return tuple(v.detach().cpu().clone() if isinstance(v, torch.Tensor) else v for v in values)


def _call_with_snapshot(fn, args, debug: bool, dump: str, what: str):
    """With debug on, a failing call leaves a CPU copy of its arguments in
    `dump` before re-raising (the reference's snapshot convention)."""
    if not debug:
        return fn(*args)
    snapshot = cpu_deep_copy_tuple(args)
    try:
        return fn(*args)
    except Exception:
        torch.save(snapshot, dump)
        print(f"\nAn error occurred in {what}. Arguments were written to {dump} for debugging.")
        raise


class _Tracer(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tracer, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                cumsum_of_points_per_triangle, number_of_points, shs, colors_precomp, opacities, scaling,
                density_factor, tracer_settings: TracerSettings):
        st = tracer_settings
        args = (ray_o, ray_d, triangles_points, sigma, num_points_per_triangle, cumsum_of_points_per_triangle,
                number_of_points, shs, st.sh_degree, colors_precomp, opacities, scaling, density_factor, st.bg,
                st.extra_params, st.rebuild_gas, st.debug)
        # every ray's first hit query, kept for the adjoint like an activation
        cache = None
        rays = int(ray_o.shape[0]) * int(ray_o.shape[1]) if ray_o.dim() >= 2 else 0
        if tracer.use_hit_cache and tracer.variant == _C._lib.TT_VARIANT_PLAIN and rays:
            cache = tracer.autograd_hit_cache(rays)
        fwd = tracer.trace_forward if cache is None else (lambda *a: tracer.trace_forward(*a, hit_cache=cache))
        res = _call_with_snapshot(fwd, args, st.debug, "snapshot_fw.dump", "forward")
        if cache is not None:
            tracer.observe_hit_cache(cache, rays)  # sizes the next forwards' pools
        color, others, gpu_time, scaling, density_factor, max_blending = res.data
        ctx.hit_cache = cache
        ctx.tracer_settings = st
        ctx.tracer = tracer
        ctx.number_of_points = number_of_points
        ctx.save_for_backward(ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                              cumsum_of_points_per_triangle, color, others, colors_precomp, opacities, shs, scaling)
        ctx.mark_non_differentiable(gpu_time, scaling, density_factor, max_blending)
        return color, gpu_time, scaling, density_factor, others, max_blending

    @staticmethod
    def backward(ctx, grad_color, _g_time, _g_scaling, _g_density, grad_others, _g_maxb):
        st = ctx.tracer_settings
        (ray_o, ray_d, triangles_points, sigma, num_points_per_triangle, cumsum_of_points_per_triangle, color,
         others, colors_precomp, opacities, shs, scaling) = ctx.saved_tensors
        if grad_color is None:
            grad_color = torch.zeros_like(color)
        if grad_others is None:
            grad_others = torch.zeros_like(others)
        args = (ray_o, ray_d, st.bg, triangles_points, sigma, num_points_per_triangle,
                cumsum_of_points_per_triangle, color, others, ctx.number_of_points, shs, st.sh_degree, opacities,
                grad_color, grad_others, scaling, st.debug)
        use_cols = shs.numel() == 0 and colors_precomp.numel() > 0  # precomputed colours in place of SH
        cache = ctx.hit_cache

        def fn(*a):
            return ctx.tracer.trace_backward(*a, colors_precomp=colors_precomp if use_cols else None,
                                             hit_cache=cache)

        res = _call_with_snapshot(fn, args, st.debug, "snapshot_bw.dump", "backward")
        ctx.hit_cache = None
        grad_triangles, grad_sigma, grad_opacities, grad_sh = res.data
        grad_cols = res.dL_dcolors.reshape(colors_precomp.shape) if use_cols else None
        return (
            None,  # tracer
            None,  # ray_o
            None,  # ray_d
            grad_triangles.reshape(triangles_points.shape),
            grad_sigma.reshape(sigma.shape),
            None,  # num_points_per_triangle
            None,  # cumsum_of_points_per_triangle
            None,  # number_of_points
            grad_sh if not use_cols else None,
            grad_cols,  # colors_precomp (the reference returns None: it never reads them)
            grad_opacities,
            None,  # scaling
            None,  # density_factor
            None,  # tracer_settings
        )


class Tracer(nn.Module):
    """``Tracer(forward_ptx, backward_ptx)``: the names select the program as
    in the reference ("forward.ptx", "reflect.ptx", "refract.ptx",
    "envlight.ptx" / "backward.ptx"); nothing is read from disk."""

    def __init__(self, forwad_ptx="forward.ptx", backward_ptx="backward.ptx", tmin_inclusive: bool = True,
                 exact_adjoint: bool = False, hit_cache: bool = True, reference_arithmetic: bool = False) -> None:
        """hit_cache (no reference counterpart): the forward keeps its
        k-closest queries in a device buffer held by the autograd graph ((k + 1)
        * 8 bytes a ray for the first ones, plus a pool of a quarter of that for
        later ones) and the backward replays them instead of traversing the BVH
        again; the gradients are the same either way.

        reference_arithmetic (no reference counterpart): evaluate each hit's
        window function in the reference's own FP32 arithmetic (hit point
        o + t d) instead of from an FP64 ray/plane solve, to reproduce the
        reference's numbers; the semantics are the same."""
        super().__init__()
        self.tracer = _C.OptixTracer("", forwad_ptx, backward_ptx, tmin_inclusive=tmin_inclusive,
                                     exact_adjoint=exact_adjoint, reference_arithmetic=reference_arithmetic)
        self.tracer.use_hit_cache = bool(hit_cache)

    def forward(self, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle, cumsum_of_points_per_triangle,
                number_of_points, opacities, scaling, density_factor, shs, colors_precomp,
                tracer_settings: TracerSettings):
        if (shs is None) == (colors_precomp is None):
            raise Exception("Please provide excatly one of either SHs or precomputed colors!")
        dev = ray_o.device
        if shs is None:
            shs = torch.empty(0, device=dev)
        if colors_precomp is None:
            colors_precomp = torch.empty(0, device=dev)
        return _Tracer.apply(self.tracer, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                             cumsum_of_points_per_triangle, number_of_points, shs, colors_precomp, opacities, scaling,
                             density_factor, tracer_settings)

    def set_proposal(self, proposal, margin_near=None, margin_far=None, far_cap=None):
        """Clips the traversal of the forward and backward passes to the
        intervals of a trained proposal network (None: plain traversal)."""
        self.tracer.set_proposal(proposal, margin_near, margin_far, far_cap)
