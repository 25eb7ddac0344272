"""Differentiable secondary-ray rendering: dielectric triangles (material 1)
reflect and refract rays, up to `max_depth` bounces, and rays that leave the
scene see a lat-long environment map. No counterpart in the reference, whose
reflect / refract / envlight programs bend rays only at one analytic sphere
and have no adjoint. The passes run on the library's device ray queue
(tt_forward_secondary / tt_backward_secondary)."""
from __future__ import annotations

import torch
import torch.nn as nn

from . import _C


class _Secondary(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tracer, ray_o, ray_d, triangles_points, sigma, num_points, cumsum, P, opacities, shs,
                sh_degree, material, ior, env, max_depth, rebuild_gas):
        scaling = torch.zeros(P, device=ray_o.device)
        density = torch.zeros(P, device=ray_o.device)
        color, others, max_blending = tracer.trace_forward_secondary(
            ray_o, ray_d, triangles_points, sigma, num_points, cumsum, P, shs, sh_degree, opacities, scaling,
            density, material, ior, env, max_depth, rebuild_gas)
        ctx.tracer, ctx.P, ctx.sh_degree, ctx.max_depth = tracer, P, sh_degree, max_depth
        ctx.save_for_backward(ray_o, ray_d, triangles_points, sigma, num_points, cumsum, opacities, shs, material,
                              ior, env, color, others)
        ctx.mark_non_differentiable(others, max_blending, scaling, density)
        return color, others, max_blending, scaling, density

    @staticmethod
    def backward(ctx, g_color, g_others, *_):
        (ray_o, ray_d, verts, sigma, num_points, cumsum, opacities, shs, material, ior, env, color,
         others) = ctx.saved_tensors
        g_color = torch.zeros_like(color) if g_color is None else g_color.contiguous()
        g_others = torch.zeros_like(others) if g_others is None else g_others.contiguous()
        want_material = ctx.needs_input_grad[12] or ctx.needs_input_grad[13]
        grads = ctx.tracer.trace_backward_secondary(
            ray_o, ray_d, verts, sigma, num_points, cumsum, color, others, ctx.P, shs, ctx.sh_degree, opacities,
            g_color, g_others, material, ior, env, ctx.max_depth, material_grads=want_material)
        d_tri, d_sigma, d_opac, d_sh = grads[:4]
        d_ior = grads[5].reshape(ior.shape) if want_material and ctx.needs_input_grad[12] else None
        d_env = grads[4].reshape(env.shape) if want_material and ctx.needs_input_grad[13] else None
        return (None, None, None, d_tri.reshape(verts.shape), d_sigma.reshape(sigma.shape), None, None, None,
                d_opac.reshape(opacities.shape), d_sh, None, None, d_ior, d_env, None, None)


class SecondaryTracer(nn.Module):
    """forward(ray_o, ray_d, triangles_points, sigma, num_points, cumsum, P,
    opacities, shs, material, ior, env) -> (color, others, max_blending,
    scaling, density_factor); gradients flow to the vertices, sigma,
    opacities and SH coefficients, and, when they require it, to the
    environment map and the IOR (through the Fresnel share of each
    refracting hit; the bent directions are held constant, as the spawn
    geometry is for every input)."""

    def __init__(self, sh_degree=3, max_depth=2, exact_adjoint=False):
        super().__init__()
        # exact_adjoint: the full chain rule of the window function (vertex
        # gradients included) for every triangle; the spawn geometry stays
        # constant
        self.tracer = _C.OptixTracer("", "forward.ptx", "backward.ptx", exact_adjoint=exact_adjoint)
        self.sh_degree, self.max_depth = sh_degree, max_depth
        self._built = False

    def forward(self, ray_o, ray_d, triangles_points, sigma, num_points, cumsum, P, opacities, shs, material, ior,
                env):
        rebuild = 1 if self._built else 0
        self._built = True
        return _Secondary.apply(self.tracer, ray_o, ray_d, triangles_points, sigma, num_points, cumsum, P,
                                opacities, shs, self.sh_degree, material, ior, env, self.max_depth, rebuild)
