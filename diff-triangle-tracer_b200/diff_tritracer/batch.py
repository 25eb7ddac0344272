"""Batched camera views of uneven resolution, captured in a CUDA graph.

`ViewBatch` traces a fixed set of views (each its own [H, W] image, up to 32)
through ONE persistent forward launch and ONE adjoint launch per step
(tt_forward_views / tt_backward_views). With `graph=True` the step - BVH refit
to the current vertices, forward, adjoint - is recorded once into a CUDA graph
and replayed, so a training step costs one graph launch on the host. With
`hit_cache=True` the forward keeps its k-closest queries in a static buffer
and the adjoint replays them instead of traversing again; the first step
(and every `fit_hit_cache()` call) grows that buffer's pool until one
forward's later queries all fit, so deep scenes replay every query. Rays and
upstream gradients are copied into the batch's static buffers before replay;
the scene tensors must keep their storage between steps (optimisers update
them in place).
"""

from __future__ import annotations

import torch

from ._C import OptixTracer


class ViewBatch:
    def __init__(self, tracer: OptixTracer, shapes, scene: dict, sh_degree: int, bg: torch.Tensor,
                 graph: bool = True, hit_cache: bool = True):
        """shapes: [(H, W)] per view. scene: dict with triangles_points, sigma,
        num_points_per_triangle, cumsum_of_points_per_triangle, number_of_points,
        shs, opacities, scaling, density_factor (device tensors)."""
        if not 1 <= len(shapes) <= 32:
            raise RuntimeError("a batch holds 1 to 32 views")
        self.tracer = tracer
        self.scene = scene
        self.sh_degree = sh_degree
        self.bg = bg
        dev = tracer.device
        f32 = dict(dtype=torch.float32, device=dev)
        self.rays = [(torch.zeros((H, W, 3), **f32), torch.zeros((H, W, 3), **f32)) for H, W in shapes]
        self.outputs = [(torch.zeros((3, H, W), **f32), torch.zeros((7, H, W), **f32)) for H, W in shapes]
        self.upstream = [(torch.zeros((3, H, W), **f32), torch.zeros((7, H, W), **f32)) for H, W in shapes]
        P = int(scene["number_of_points"])
        self.max_blending = torch.zeros((P,), **f32)
        V = scene["triangles_points"].numel() // 3
        M = scene["shs"].shape[1]
        self.grads = (torch.zeros((V, 3), **f32), torch.zeros_like(scene["sigma"]),
                      torch.zeros_like(scene["opacities"]), torch.zeros((P, M, 3), **f32))
        self.num_rays = sum(H * W for H, W in shapes)
        # sized for 32-hit queries, so it serves every traversal configuration
        self.hit_cache = tracer.new_hit_cache(self.num_rays, k=32) if hit_cache else None
        self._fitted = not hit_cache
        self.graph = None
        # the first pass builds the BVH outside any capture
        self._forward(0)
        self._backward()
        torch.cuda.synchronize()
        self._use_graph = graph
        self._capture()

    def _capture(self):
        self.graph = None
        if self._use_graph:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                self._forward(1)
                self._backward()
            self.graph = graph

    def fit_hit_cache(self, rounds: int = 4):
        """Runs forwards over the current rays and grows the hit cache's pool
        until all of one forward's later queries fit (a ray stops asking after
        its first refusal, so an overflow may take a few rounds to size). The
        graph is recorded again if the buffer changed. Synchronises; returns
        the last forward's pool usage (see OptixTracer.hit_cache_usage)."""
        self._fitted = True
        if self.hit_cache is None:
            return None
        grown = False
        for _ in range(rounds):
            self._forward(1)
            use = self.tracer.hit_cache_usage(self.hit_cache)
            if use["pool_used"] <= use["pool_cap"]:
                break
            self.hit_cache = None  # release the old buffer first
            self.hit_cache = self.tracer.new_hit_cache(self.num_rays, k=32, pool=int(use["pool_used"] * 1.25) + 1024)
            grown = True
        if grown:
            self._capture()
        return use

    def _forward(self, rebuild_gas):
        s = self.scene
        self.tracer.trace_forward_views(self.rays, s["triangles_points"], s["sigma"], s["num_points_per_triangle"],
                                        s["cumsum_of_points_per_triangle"], s["number_of_points"], s["shs"],
                                        self.sh_degree, s["opacities"], s["scaling"], s["density_factor"], self.bg,
                                        rebuild_gas, outputs=self.outputs, max_blending=self.max_blending,
                                        hit_cache=self.hit_cache)

    def _backward(self):
        s = self.scene
        self.tracer.trace_backward_views(self.rays, self.outputs, self.upstream, s["triangles_points"], s["sigma"],
                                         s["num_points_per_triangle"], s["cumsum_of_points_per_triangle"],
                                         s["number_of_points"], s["shs"], self.sh_degree, s["opacities"], self.bg,
                                         grads=self.grads, hit_cache=self.hit_cache)

    def set_rays(self, rays):
        for (ro, rd), (so, sd) in zip(rays, self.rays):
            so.copy_(ro, non_blocking=True)
            sd.copy_(rd, non_blocking=True)

    def set_cameras(self, cameras):
        """Generates the views' rays on the device from pinhole cameras
        (scenes.Camera, one per view, of the batch's shapes) into the static
        ray buffers: one launch, no host copy (OptixTracer.camera_rays)."""
        self.tracer.camera_rays(cameras, outputs=self.rays)

    def set_upstream(self, upstream):
        for (g, go), (sg, sgo) in zip(upstream, self.upstream):
            sg.copy_(g, non_blocking=True)
            sgo.copy_(go, non_blocking=True)

    def step(self):
        """Refit + forward + adjoint over all views; results in .outputs,
        .max_blending and .grads. The first step fits the hit cache to the
        rays (fit_hit_cache) and synchronises."""
        if not self._fitted:
            self.fit_hit_cache()
        if self.graph is not None:
            self.graph.replay()
        else:
            self._forward(1)
            self._backward()
