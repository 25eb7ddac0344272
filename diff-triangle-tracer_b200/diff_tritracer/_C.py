"""Host-side mirror of the reference's pybind11 module ``_C`` (ext.cpp:11-27):
``OptixTracer`` with ``build_tri_accel``, ``trace_forward`` and
``trace_backward``, returning objects with a ``.data`` tuple, over the C ABI of
libtritracer.so. Tensors are handed over as raw device pointers on the
current torch stream; no OptiX is involved.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import lib, check

# the PTX names the reference loads select a raygen program here
_VARIANTS = {
    "forward.ptx": _lib.TT_VARIANT_PLAIN,
    "reflect.ptx": _lib.TT_VARIANT_REFLECT,
    "refract.ptx": _lib.TT_VARIANT_REFRACT,
    "envlight.ptx": _lib.TT_VARIANT_ENVLIGHT,
}


class FwdTraceResult:
    """tracer.h:59-61: data = (color, others, gpu_time, scaling, density_factor, max_blending)."""

    def __init__(self, data):
        self.data = data


class BwdTraceResult:
    """tracer.h:63-65: data = (dL_dtriangle, dL_dsigma, dL_dopacity, dL_dsh)."""

    def __init__(self, data):
        self.data = data


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def _set_cache(a, hit_cache, device):
    """Puts an optional hit-cache buffer (uint8 device tensor) into an argument block."""
    if hit_cache is None:
        a.hit_cache, a.hit_cache_bytes = ctypes.c_void_p(0), 0
        return
    if not isinstance(hit_cache, torch.Tensor) or hit_cache.device != device or not hit_cache.is_contiguous():
        raise RuntimeError("hit_cache must be a contiguous tensor on the tracer's device (new_hit_cache)")
    a.hit_cache, a.hit_cache_bytes = _ptr(hit_cache), hit_cache.numel() * hit_cache.element_size()


def _f32(t, name, device):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be float32, got {t.dtype}")
    if t.device != device:
        raise RuntimeError(f"{name} must be on {device}, got {t.device}")
    return t.contiguous()


def _i32(t, name, device):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if t.dtype != torch.int32:
        raise RuntimeError(f"{name} must be int32, got {t.dtype}")
    if t.device != device:
        raise RuntimeError(f"{name} must be on {device}, got {t.device}")
    return t.contiguous()


class OptixTracer:
    """Drop-in for the reference's ``_C.OptixTracer(pkgDir[, forward, backward])``
    (tracer.h:67-126). ``pkgDir`` is accepted for signature compatibility and
    unused; the two names select the program (forward.ptx, reflect.ptx,
    refract.ptx, envlight.ptx / backward.ptx)."""

    def __init__(self, pkg_dir: str = "", forward: str = "forward.ptx", backward: str = "backward.ptx",
                 tmin_inclusive: bool = True, traversal: str = "auto", exact_adjoint: bool = False,
                 reference_arithmetic: bool = False):
        if forward not in _VARIANTS:
            raise RuntimeError(f"unknown forward program {forward!r}; expected one of {sorted(_VARIANTS)}")
        if backward != "backward.ptx":
            raise RuntimeError(f"unknown backward program {backward!r}; expected 'backward.ptx'")
        if not torch.cuda.is_available():
            raise RuntimeError("OptixTracer needs a CUDA device")
        self.variant = _VARIANTS[forward]
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.use_hit_cache = False  # set by diff_tritracer.Tracer (its autograd path passes a hit cache)
        self._pool_frac = 0.25  # autograd hit caches: pool size as a fraction of the rays (observe_hit_cache)
        self._cache_calls = 0
        cfg = _lib.TtConfig()
        cfg.variant = self.variant
        cfg.tmin_inclusive = 1 if tmin_inclusive else 0
        modes = {"auto": _lib.TT_TRAVERSAL_AUTO, "packets": _lib.TT_TRAVERSAL_PACKETS, "lanes": _lib.TT_TRAVERSAL_LANES}
        if traversal not in modes:
            raise RuntimeError(f"traversal must be one of {sorted(modes)}")
        cfg.traversal = modes[traversal]
        cfg.exact_adjoint = 1 if exact_adjoint else 0
        # the reference's own FP32 arithmetic for the window function (see
        # tt_config.reference_arithmetic); default: FP64 ray/plane solve
        cfg.reference_arithmetic = 1 if reference_arithmetic else 0
        h = ctypes.c_void_p(0)
        rc = lib.tt_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != _lib.TT_OK:
            raise _lib.TracerError(rc, f"OptixTracer construction failed (tt_create returned {rc})")
        self._h = h
        self._destroy = lib.tt_destroy
        self._keep = ()
        self._proposal = None
        self._proposal_args = (None, None, None)

    def __del__(self):
        # the bound function, not the module global: at interpreter exit the
        # module's globals may already be cleared when this runs
        h, destroy = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and destroy is not None:
            destroy(h)
            self._h = None

    # ------------------------------------------------------------------
    def build_tri_accel(self, triangles_points, cumsum_of_points_per_triangle, number_of_points, rebuild=True):
        """pipeline.cpp:206-265 (BUILD when `rebuild`, UPDATE otherwise)."""
        dev = self.device
        verts = _f32(triangles_points, "triangles_points", dev)
        cumsum = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        mode = 0 if rebuild else 1
        check(self._h, lib.tt_build(self._h, _ptr(verts), verts.numel() // 3, _ptr(cumsum), int(number_of_points),
                                    mode, _stream()))

    def save_bvh(self, path=None):
        """Serialises the acceleration structure's topology (bytes; also
        written to `path` when given). No reference counterpart."""
        n = ctypes.c_ulonglong(0)
        check(self._h, lib.tt_bvh_save(self._h, None, 0, ctypes.byref(n), _stream()))
        out = bytearray(n.value)
        if n.value:
            check(self._h, lib.tt_bvh_save(self._h, (ctypes.c_char * n.value).from_buffer(out), n.value,
                                           ctypes.byref(n), _stream()))
        blob = bytes(out)
        if path is not None:
            with open(path, "wb") as f:
                f.write(blob)
        return blob

    def load_bvh(self, blob_or_path, triangles_points, cumsum_of_points_per_triangle, number_of_points):
        """Restores a saved topology and refits it to these vertices (the
        same triangles), instead of building: the next trace may use
        rebuild_gas = 2 (keep) or 1 (refit)."""
        blob = blob_or_path
        if not isinstance(blob, (bytes, bytearray)):
            with open(blob_or_path, "rb") as f:
                blob = f.read()
        verts = _f32(triangles_points, "triangles_points", self.device)
        cumsum = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", self.device)
        # the C side only reads the blob: pass the bytes object's own storage
        src = ctypes.c_char_p(bytes(blob) if isinstance(blob, bytearray) else blob)
        check(self._h, lib.tt_bvh_load(self._h, ctypes.cast(src, ctypes.c_void_p), len(blob), _ptr(verts),
                                       verts.numel() // 3, _ptr(cumsum), int(number_of_points), _stream()))
        self._keep = (verts, cumsum)

    def new_hit_cache(self, rays, k=None, pool=None):
        """A device buffer for the hit cache of `rays` rays: sized for the
        current traversal configuration (tt_hit_cache_bytes_pool), or for
        queries of `k` hits (k = 32 fits every configuration), with room for
        `pool` later queries (default: a quarter of the rays). No reference
        counterpart."""
        rays = int(rays)
        pool = (rays + 3) // 4 if pool is None else int(pool)
        n = lib.tt_hit_cache_bytes_pool(self._h, rays, pool)
        if k is not None:
            n = max(n, 32 + (int(k) + 1) * 8 * rays + (int(k) + 2) * 8 * pool)
        return torch.empty((n,), dtype=torch.uint8, device=self.device)

    def camera_rays(self, cameras, outputs=None):
        """Primary rays of pinhole cameras (diff_tritracer.scenes.Camera: origin,
        forward/right/up basis, H, W, vertical fov_deg) generated on the device
        in one launch (tt_camera_rays), bit for bit the rays of
        scenes.camera_rays. Returns [(ray_o, ray_d)] per camera, [H, W, 3]
        each, written into `outputs` when given. No reference counterpart: the
        reference's callers build the ray tensors themselves."""
        cams = list(cameras)
        if outputs is None:
            outputs = [(torch.empty((c.H, c.W, 3), dtype=torch.float32, device=self.device),
                        torch.empty((c.H, c.W, 3), dtype=torch.float32, device=self.device)) for c in cams]
        if len(outputs) != len(cams):
            raise RuntimeError("one (ray_o, ray_d) pair per camera")
        arr = (_lib.TtCamera * max(len(cams), 1))()
        for a, c, (ro, rd) in zip(arr, cams, outputs):
            for t in (ro, rd):
                if t.dtype != torch.float32 or t.device != self.device or not t.is_contiguous() \
                        or tuple(t.shape) != (c.H, c.W, 3):
                    raise RuntimeError("camera ray outputs must be contiguous float32 [H, W, 3] on the tracer's device")
            for name in ("origin", "forward", "right", "up"):
                getattr(a, name)[:] = [float(x) for x in getattr(c, name)]
            a.tan_half_fov = float(np.tan(np.deg2rad(c.fov_deg) / 2.0))  # as scenes.camera_rays
            a.H, a.W = int(c.H), int(c.W)
            a.ray_o, a.ray_d = _ptr(ro), _ptr(rd)
        check(self._h, lib.tt_camera_rays(self._h, arr, len(cams), _stream()))
        return outputs

    def autograd_hit_cache(self, rays):
        """The autograd module's hit cache for one forward: its pool holds the
        fraction of the rays that earlier forwards' later queries needed
        (observe_hit_cache), a quarter at first."""
        return self.new_hit_cache(rays, pool=max(int(self._pool_frac * rays), 1))

    def observe_hit_cache(self, hit_cache, rays):
        """After the first two autograd forwards, and every 1024th after that,
        reads how many later queries the pool was asked for (one stream
        synchronisation) and grows the pool fraction when they did not fit.
        The calls in between read nothing."""
        n = self._cache_calls
        self._cache_calls += 1
        if n >= 2 and n % 1024:
            return
        use = self.hit_cache_usage(hit_cache)
        if use["pool_used"] > use["pool_cap"]:
            self._pool_frac = max(self._pool_frac, 1.25 * use["pool_used"] / max(int(rays), 1))

    def hit_cache_usage(self, hit_cache):
        """The header of a hit cache a forward has filled (synchronises the
        current stream): {"k", "pool_cap", "pool_used"}. pool_used > pool_cap
        means some later queries were not stored and the adjoint traverses
        again for them; the count is then a lower bound on what the pool
        needs (a ray stops asking after its first refusal)."""
        k, cap, used = ctypes.c_int(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
        check(self._h, lib.tt_hit_cache_usage(self._h, ctypes.c_void_p(hit_cache.data_ptr()), _stream(),
                                              ctypes.byref(k), ctypes.byref(cap), ctypes.byref(used)))
        return {"k": k.value, "pool_cap": cap.value, "pool_used": used.value}

    def trace_forward(self, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                      cumsum_of_points_per_triangle, number_of_points, shs, sh_degree, colors_precomp, opacities,
                      scaling, density_factor, bg_color, extra, rebuild_gas_opt, debug, hit_cache=None):
        """tracer.cpp:16-142: returns FwdTraceResult((color [3,H,W], others [7,H,W],
        gpu_time [1], scaling, density_factor, max_blending [P])). With
        `hit_cache` (a new_hit_cache(H * W) buffer) the forward also stores every
        ray's k-closest queries there for trace_backward."""
        dev = self.device
        P = int(number_of_points)
        ro = _f32(ray_o, "ray_o", dev)
        rd = _f32(ray_d, "ray_d", dev)
        if ro.dim() < 2 or ro.shape != rd.shape or ro.shape[-1] != 3:
            raise RuntimeError("ray_o / ray_d must both be [H, W, 3]")
        H, W = int(ro.shape[0]), int(ro.shape[1])
        verts = _f32(triangles_points, "triangles_points", dev)
        sig = _f32(sigma, "sigma", dev)
        npts = _i32(num_points_per_triangle, "num_points_per_triangle", dev)
        cums = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        sh = _f32(shs, "shs", dev)
        M = int(sh.shape[1]) if sh.dim() >= 2 and sh.shape[0] != 0 else 0
        opac = _f32(opacities, "opacities", dev)
        bg = _f32(bg_color, "bg_color", dev)
        ex = extra.to(device=dev, dtype=torch.float32).contiguous() if isinstance(extra, torch.Tensor) else None
        if ex is not None and ex.numel() == 0:
            ex = None
        # scaling / density_factor are updated in place and returned
        sc = _f32(scaling, "scaling", dev)
        de = _f32(density_factor, "density_factor", dev)
        out_color = torch.empty((3, H, W), dtype=torch.float32, device=dev)
        out_others = torch.empty((7, H, W), dtype=torch.float32, device=dev)
        max_blending = torch.empty((P,), dtype=torch.float32, device=dev)
        ms = ctypes.c_float(0.0)
        a = _lib.TtFwdArgs()
        a.H, a.W = H, W
        a.ray_o, a.ray_d = _ptr(ro), _ptr(rd)
        a.vertices, a.num_vertices = _ptr(verts), verts.numel() // 3
        a.num_points, a.cumsum, a.P = _ptr(npts), _ptr(cums), P
        a.shs, a.sh_degree, a.M = (_ptr(sh) if sh.numel() else ctypes.c_void_p(0)), int(sh_degree), M
        cp = None
        if sh.numel() == 0 and isinstance(colors_precomp, torch.Tensor) and colors_precomp.numel():
            cp = _f32(colors_precomp, "colors_precomp", dev)  # [P, 3] in place of SH
        a.colors_precomp = _ptr(cp) if cp is not None else ctypes.c_void_p(0)
        a.opacities, a.sigma = _ptr(opac), _ptr(sig)
        a.scaling, a.density_factor = _ptr(sc), _ptr(de)
        a.bg = _ptr(bg)
        a.extra, a.extra_len = (_ptr(ex), ex.numel()) if ex is not None else (ctypes.c_void_p(0), 0)
        a.rebuild_gas, a.debug = int(rebuild_gas_opt), 1 if debug else 0
        a.out_color, a.out_others, a.max_blending = _ptr(out_color), _ptr(out_others), _ptr(max_blending)
        a.gpu_time_ms = ctypes.pointer(ms)
        _set_cache(a, hit_cache, dev)
        if self._proposal is not None:
            v = _lib.TtView()
            v.H, v.W, v.ray_o, v.ray_d = H, W, a.ray_o, a.ray_d
            v.out_color, v.out_others = a.out_color, a.out_others
            iv = self._intervals(ro, rd)
            v.interval = _ptr(iv)
            check(self._h, lib.tt_forward_views(self._h, ctypes.byref(a), ctypes.byref(v), 1, _stream()))
        else:
            iv = None
            check(self._h, lib.tt_forward(self._h, ctypes.byref(a), _stream()))
        if sc.data_ptr() != scaling.data_ptr():
            scaling.copy_(sc.view_as(scaling))
        if de.data_ptr() != density_factor.data_ptr():
            density_factor.copy_(de.view_as(density_factor))
        gpu_time = torch.zeros((1,), dtype=torch.float32, device=dev)
        if debug:
            gpu_time.fill_(ms.value)
        # the arrays the kernels read must outlive the asynchronous launch
        self._keep = (ro, rd, verts, sig, npts, cums, sh, opac, bg, ex, sc, de, iv, cp, hit_cache)
        return FwdTraceResult((out_color, out_others, gpu_time, scaling, density_factor, max_blending))

    def trace_backward(self, ray_o, ray_d, background, triangles_points, sigma, num_points_per_triangle,
                       cumsum_of_points_per_triangle, colors, others, number_of_points, shs, sh_degree, opacities,
                       dL_dpixels, dL_dothers, scaling, debug, colors_precomp=None, hit_cache=None):
        """tracer.cpp:144-228: returns BwdTraceResult((dL_dtriangle [V,3],
        dL_dsigma like sigma, dL_dopacity like opacities, dL_dsh [P,M,3])).
        With empty shs and colors_precomp [P, 3] (the forward's colours) the
        result also carries .dL_dcolors [P, 3]. `hit_cache`: the buffer the
        forward of these rays filled; the adjoint replays it where still valid
        (same results either way)."""
        dev = self.device
        P = int(number_of_points)
        ro = _f32(ray_o, "ray_o", dev)
        rd = _f32(ray_d, "ray_d", dev)
        H, W = int(ro.shape[0]), int(ro.shape[1])
        verts = _f32(triangles_points, "triangles_points", dev)
        sig = _f32(sigma, "sigma", dev)
        npts = _i32(num_points_per_triangle, "num_points_per_triangle", dev)
        cums = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        col = _f32(colors, "colors", dev)
        oth = _f32(others, "others", dev)
        sh = _f32(shs, "shs", dev)
        M = int(sh.shape[1]) if sh.dim() >= 2 and sh.shape[0] != 0 else 0
        opac = _f32(opacities, "opacities", dev)
        g = _f32(dL_dpixels, "dL_dpixels", dev)
        go = _f32(dL_dothers, "dL_dothers", dev)
        bg = _f32(background, "background", dev)
        V = verts.numel() // 3
        dL_dtriangle = torch.empty((V, 3), dtype=torch.float32, device=dev)
        dL_dsigma = torch.empty_like(sigma, memory_format=torch.contiguous_format)
        dL_dopacity = torch.empty_like(opacities, memory_format=torch.contiguous_format)
        dL_dsh = torch.empty((P, M, 3), dtype=torch.float32, device=dev)
        a = _lib.TtBwdArgs()
        a.H, a.W = H, W
        a.ray_o, a.ray_d, a.bg = _ptr(ro), _ptr(rd), _ptr(bg)
        a.vertices, a.num_vertices = _ptr(verts), V
        a.sigma, a.num_points, a.cumsum = _ptr(sig), _ptr(npts), _ptr(cums)
        a.colors, a.others, a.P = _ptr(col), _ptr(oth), P
        a.shs, a.sh_degree, a.M = (_ptr(sh) if sh.numel() else ctypes.c_void_p(0)), int(sh_degree), M
        cp = dcols = None
        if sh.numel() == 0 and isinstance(colors_precomp, torch.Tensor) and colors_precomp.numel():
            cp = _f32(colors_precomp, "colors_precomp", dev)
            dcols = torch.empty((P, 3), dtype=torch.float32, device=dev)
            a.colors_precomp, a.dL_dcolors = _ptr(cp), _ptr(dcols)
        a.opacities, a.dL_dpixels, a.dL_dothers = _ptr(opac), _ptr(g), _ptr(go)
        a.scaling = ctypes.c_void_p(0)
        a.debug = 1 if debug else 0
        a.dL_dtriangle, a.dL_dsigma = _ptr(dL_dtriangle), _ptr(dL_dsigma)
        a.dL_dopacity, a.dL_dsh = _ptr(dL_dopacity), _ptr(dL_dsh)
        a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
        _set_cache(a, hit_cache, dev)
        if self._proposal is not None:
            v = _lib.TtView()
            v.H, v.W, v.ray_o, v.ray_d = H, W, a.ray_o, a.ray_d
            v.colors, v.others, v.dL_dpixels, v.dL_dothers = a.colors, a.others, a.dL_dpixels, a.dL_dothers
            iv = self._intervals(ro, rd)
            v.interval = _ptr(iv)
            check(self._h, lib.tt_backward_views(self._h, ctypes.byref(a), ctypes.byref(v), 1, _stream()))
        else:
            iv = None
            check(self._h, lib.tt_backward(self._h, ctypes.byref(a), _stream()))
        self._keep = (ro, rd, verts, sig, npts, cums, col, oth, sh, opac, g, go, bg, iv, cp, hit_cache)
        res = BwdTraceResult((dL_dtriangle, dL_dsigma, dL_dopacity, dL_dsh))
        res.dL_dcolors = dcols
        return res

    # ------------------------------------------------------------------
    def set_proposal(self, proposal, margin_near=None, margin_far=None, far_cap=None):
        """Clips every plain trace_forward / trace_backward of this handle to
        the intervals of a trained `diff_tritracer.proposal.Proposal` (None:
        back to the plain traversal). The network runs on the same rays in
        the forward and in the adjoint, so both visit the same hits. No
        reference counterpart."""
        if proposal is not None and self.variant != _lib.TT_VARIANT_PLAIN:
            raise RuntimeError("proposed intervals are for the plain program only")
        self._proposal = proposal
        self._proposal_args = (margin_near, margin_far, far_cap)

    def _intervals(self, ro, rd):
        mn, mf, cap = self._proposal_args
        return self._proposal.intervals([(ro, rd)], mn, mf, cap)[0]

    def set_traversal(self, traversal: str = "auto", k: int = 16, stack_depth: int = 32):
        """Switches the traversal configuration (the BVH is kept)."""
        modes = {"auto": _lib.TT_TRAVERSAL_AUTO, "packets": _lib.TT_TRAVERSAL_PACKETS, "lanes": _lib.TT_TRAVERSAL_LANES}
        check(self._h, lib.tt_set_traversal(self._h, modes[traversal], int(k), int(stack_depth)))

    def set_split_forward(self, on: bool = True):
        """With a hit cache, run the plain forward as a traversal-only pass
        that stores every query followed by a shading pass that replays them
        (default), or as one fused kernel (False). The results are the same."""
        check(self._h, lib.tt_set_option(self._h, _lib.TT_OPT_SPLIT_FORWARD, 1 if on else 0))

    def forward_pass_times(self):
        """(collecting pass ms, shading pass ms) of the last forward run with
        debug=True (0 for the first when the forward was fused)."""
        a, b = ctypes.c_float(0.0), ctypes.c_float(0.0)
        check(self._h, lib.tt_forward_pass_times(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_collect_queries(self, n: int = 2):
        """Queries per ray the split forward's traversal-only pass stores at
        most (0: all of the march's); the shading pass traverses the rest."""
        check(self._h, lib.tt_set_option(self._h, _lib.TT_OPT_COLLECT_QUERIES, int(n)))

    def set_work_counters(self, on: bool = True):
        """Count node visits and triangle tests into stats() (off by default:
        the counts cost the packet traversal ~4 % of its time)."""
        check(self._h, lib.tt_set_option(self._h, _lib.TT_OPT_WORK_COUNTERS, 1 if on else 0))

    def set_sort_secondary(self, on: bool = True):
        """Trace each level of spawned secondary rays sorted by direction
        (octahedral bins) and origin (default) or in spawn order (False). The results
        are the same."""
        check(self._h, lib.tt_set_option(self._h, _lib.TT_OPT_SORT_SECONDARY, 1 if on else 0))

    def _scene_fwd_args(self, triangles_points, sigma, num_points_per_triangle, cumsum_of_points_per_triangle,
                        number_of_points, shs, sh_degree, opacities, scaling, density_factor, bg_color,
                        rebuild_gas_opt, max_blending):
        dev = self.device
        verts = _f32(triangles_points, "triangles_points", dev)
        sig = _f32(sigma, "sigma", dev)
        npts = _i32(num_points_per_triangle, "num_points_per_triangle", dev)
        cums = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        sh = _f32(shs, "shs", dev)
        opac = _f32(opacities, "opacities", dev)
        bg = _f32(bg_color, "bg_color", dev)
        if not (scaling.is_contiguous() and density_factor.is_contiguous()):
            raise RuntimeError("scaling and density_factor must be contiguous for batched calls")
        a = _lib.TtFwdArgs()
        a.vertices, a.num_vertices = _ptr(verts), verts.numel() // 3
        a.num_points, a.cumsum, a.P = _ptr(npts), _ptr(cums), int(number_of_points)
        a.shs, a.sh_degree, a.M = _ptr(sh), int(sh_degree), int(sh.shape[1]) if sh.dim() >= 2 and sh.shape[0] else 0
        a.opacities, a.sigma = _ptr(opac), _ptr(sig)
        a.scaling, a.density_factor = _ptr(scaling), _ptr(density_factor)
        a.bg = _ptr(bg)
        a.rebuild_gas = int(rebuild_gas_opt)
        a.max_blending = _ptr(max_blending)
        a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
        return a, (verts, sig, npts, cums, sh, opac, bg)

    # ------------------------------------------------------------------ secondary rays
    def _secondary(self, material, ior, env, max_depth):
        dev = self.device
        mat = _i32(material, "material", dev)
        io = _f32(ior, "ior", dev)
        ev = _f32(env, "env", dev)
        if ev.dim() != 3 or ev.shape[2] != 3:
            raise RuntimeError("env must be [env_h, env_w, 3]")
        sec = _lib.TtSecondary(_ptr(mat), _ptr(io), _ptr(ev), int(ev.shape[0]), int(ev.shape[1]), int(max_depth))
        return sec, (mat, io, ev)

    def trace_forward_secondary(self, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                                cumsum_of_points_per_triangle, number_of_points, shs, sh_degree, opacities, scaling,
                                density_factor, material, ior, env, max_depth=2, rebuild_gas_opt=0, debug=False):
        """Secondary-ray passes (dielectric triangles spawn reflected and
        refracted rays up to max_depth bounces, an environment map lights
        escaping rays). Returns (color [3,H,W], others [7,H,W], max_blending
        [P]); scaling and density_factor are updated in place."""
        dev = self.device
        P = int(number_of_points)
        ro, rd = _f32(ray_o, "ray_o", dev), _f32(ray_d, "ray_d", dev)
        H, W = int(ro.shape[0]), int(ro.shape[1])
        max_blending = torch.empty((P,), dtype=torch.float32, device=dev)
        bg = torch.zeros(3, device=dev)
        a, keep = self._scene_fwd_args(triangles_points, sigma, num_points_per_triangle,
                                       cumsum_of_points_per_triangle, number_of_points, shs, sh_degree, opacities,
                                       scaling, density_factor, bg, rebuild_gas_opt, max_blending)
        color = torch.empty((3, H, W), dtype=torch.float32, device=dev)
        others = torch.empty((7, H, W), dtype=torch.float32, device=dev)
        ms = ctypes.c_float(0.0)
        a.H, a.W, a.ray_o, a.ray_d = H, W, _ptr(ro), _ptr(rd)
        a.out_color, a.out_others = _ptr(color), _ptr(others)
        a.debug = 1 if debug else 0
        a.gpu_time_ms = ctypes.pointer(ms)
        sec, skeep = self._secondary(material, ior, env, max_depth)
        check(self._h, lib.tt_forward_secondary(self._h, ctypes.byref(a), ctypes.byref(sec), _stream()))
        self._keep = keep + skeep + (ro, rd)
        self.last_gpu_time_ms = ms.value
        return color, others, max_blending

    def secondary_tree(self):
        """Test hook: (records [N, 16] float32 view of the last secondary
        forward's ray records, counts per level). Record fields: o[3],
        pixel (int bits), d[3], tau, L[3], F, w, child_r, child_t (int bits)."""
        counts = (ctypes.c_int * 3)()
        check(self._h, lib.tt_secondary_tree(self._h, None, 0, counts, _stream()))
        depth = sum(1 for c in counts[1:] if c > 0)
        R = counts[0]
        n = R * (2 ** (len(counts)) - 1)
        buf = torch.zeros((n, 16), dtype=torch.float32, device=self.device)
        check(self._h, lib.tt_secondary_tree(self._h, _ptr(buf), buf.numel() * 4, counts, _stream()))
        return buf, list(counts)

    def trace_backward_secondary(self, ray_o, ray_d, triangles_points, sigma, num_points_per_triangle,
                                 cumsum_of_points_per_triangle, colors, others, number_of_points, shs, sh_degree,
                                 opacities, dL_dpixels, dL_dothers, material, ior, env, max_depth=2,
                                 material_grads=False):
        """Adjoint of the last trace_forward_secondary (same rays and scene):
        (dL_dtriangle [V,3], dL_dsigma, dL_dopacity, dL_dsh [P,M,3]), and with
        material_grads also dL_denv [env_h, env_w, 3] and dL_dior [P] (through
        the Fresnel share; bent directions held constant)."""
        dev = self.device
        P = int(number_of_points)
        ro, rd = _f32(ray_o, "ray_o", dev), _f32(ray_d, "ray_d", dev)
        H, W = int(ro.shape[0]), int(ro.shape[1])
        verts = _f32(triangles_points, "triangles_points", dev)
        sig = _f32(sigma, "sigma", dev)
        npts = _i32(num_points_per_triangle, "num_points_per_triangle", dev)
        cums = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        col, oth = _f32(colors, "colors", dev), _f32(others, "others", dev)
        sh = _f32(shs, "shs", dev)
        M = int(sh.shape[1]) if sh.dim() >= 2 and sh.shape[0] != 0 else 0
        opac = _f32(opacities, "opacities", dev)
        g, go = _f32(dL_dpixels, "dL_dpixels", dev), _f32(dL_dothers, "dL_dothers", dev)
        V = verts.numel() // 3
        grads = (torch.empty((V, 3), dtype=torch.float32, device=dev),
                 torch.empty_like(sigma, memory_format=torch.contiguous_format),
                 torch.empty_like(opacities, memory_format=torch.contiguous_format),
                 torch.empty((P, M, 3), dtype=torch.float32, device=dev))
        bg = torch.zeros(3, device=dev)
        a = _lib.TtBwdArgs()
        a.H, a.W = H, W
        a.ray_o, a.ray_d, a.bg = _ptr(ro), _ptr(rd), _ptr(bg)
        a.vertices, a.num_vertices = _ptr(verts), V
        a.sigma, a.num_points, a.cumsum = _ptr(sig), _ptr(npts), _ptr(cums)
        a.colors, a.others, a.P = _ptr(col), _ptr(oth), P
        a.shs, a.sh_degree, a.M = _ptr(sh), int(sh_degree), M
        a.opacities, a.dL_dpixels, a.dL_dothers = _ptr(opac), _ptr(g), _ptr(go)
        a.scaling = ctypes.c_void_p(0)
        a.dL_dtriangle, a.dL_dsigma, a.dL_dopacity, a.dL_dsh = [_ptr(x) for x in grads]
        a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
        sec, skeep = self._secondary(material, ior, env, max_depth)
        if material_grads:
            grads = grads + (torch.empty((sec.env_h, sec.env_w, 3), dtype=torch.float32, device=dev),
                             torch.empty((P,), dtype=torch.float32, device=dev))
            sec.dL_denv, sec.dL_dior = _ptr(grads[4]), _ptr(grads[5])
        check(self._h, lib.tt_backward_secondary(self._h, ctypes.byref(a), ctypes.byref(sec), _stream()))
        self._keep = (ro, rd, verts, sig, npts, cums, col, oth, sh, opac, g, go, bg) + skeep
        return grads

    def trace_forward_views(self, rays, triangles_points, sigma, num_points_per_triangle,
                            cumsum_of_points_per_triangle, number_of_points, shs, sh_degree, opacities, scaling,
                            density_factor, bg_color, rebuild_gas_opt, outputs=None, max_blending=None,
                            intervals=None, records=None, hit_cache=None):
        """Forward over up to 32 views of any resolutions in one launch.
        rays: list of (ray_o, ray_d), each [H, W, 3]. Returns ([(color, others)], max_blending).
        intervals: optional per-view [2, H, W] proposed [t_near, t_far] clips (None entries allowed);
        records: optional per-view [3, H, W] outputs of (t_first, t_last, terminated) per ray;
        hit_cache: optional new_hit_cache(sum of H * W) buffer for trace_backward_views."""
        dev = self.device
        P = int(number_of_points)
        if max_blending is None:
            max_blending = torch.empty((P,), dtype=torch.float32, device=dev)
        a, keep = self._scene_fwd_args(triangles_points, sigma, num_points_per_triangle,
                                       cumsum_of_points_per_triangle, number_of_points, shs, sh_degree, opacities,
                                       scaling, density_factor, bg_color, rebuild_gas_opt, max_blending)
        vs = (_lib.TtView * len(rays))()
        outs = []
        for i, (ro, rd) in enumerate(rays):
            ro = _f32(ro, "ray_o", dev)
            rd = _f32(rd, "ray_d", dev)
            H, W = int(ro.shape[0]), int(ro.shape[1])
            if outputs is None:
                col = torch.empty((3, H, W), dtype=torch.float32, device=dev)
                oth = torch.empty((7, H, W), dtype=torch.float32, device=dev)
            else:
                col, oth = outputs[i]
            vs[i].H, vs[i].W = H, W
            vs[i].ray_o, vs[i].ray_d = _ptr(ro), _ptr(rd)
            vs[i].out_color, vs[i].out_others = _ptr(col), _ptr(oth)
            outs.append((col, oth))
            keep = keep + (ro, rd)
            keep = keep + self._interval_record(vs[i], H, W, intervals, records, i)
        _set_cache(a, hit_cache, dev)
        check(self._h, lib.tt_forward_views(self._h, ctypes.byref(a), vs, len(rays), _stream()))
        self._keep = keep + (hit_cache,)
        return outs, max_blending

    def trace_backward_views(self, rays, forward_outputs, upstream, triangles_points, sigma,
                             num_points_per_triangle, cumsum_of_points_per_triangle, number_of_points, shs,
                             sh_degree, opacities, bg_color, grads=None, intervals=None, hit_cache=None):
        """Adjoint over the views of trace_forward_views. upstream: list of
        (dL_dpixels [3,H,W], dL_dothers [7,H,W]). Returns (dL_dtriangle, dL_dsigma,
        dL_dopacity, dL_dsh) summed over the views."""
        dev = self.device
        P = int(number_of_points)
        verts = _f32(triangles_points, "triangles_points", dev)
        sig = _f32(sigma, "sigma", dev)
        npts = _i32(num_points_per_triangle, "num_points_per_triangle", dev)
        cums = _i32(cumsum_of_points_per_triangle, "cumsum_of_points_per_triangle", dev)
        sh = _f32(shs, "shs", dev)
        M = int(sh.shape[1]) if sh.dim() >= 2 and sh.shape[0] != 0 else 0
        opac = _f32(opacities, "opacities", dev)
        bg = _f32(bg_color, "bg_color", dev)
        V = verts.numel() // 3
        if grads is None:
            grads = (torch.empty((V, 3), dtype=torch.float32, device=dev),
                     torch.empty_like(sigma, memory_format=torch.contiguous_format),
                     torch.empty_like(opacities, memory_format=torch.contiguous_format),
                     torch.empty((P, M, 3), dtype=torch.float32, device=dev))
        a = _lib.TtBwdArgs()
        a.bg = _ptr(bg)
        a.vertices, a.num_vertices = _ptr(verts), V
        a.sigma, a.num_points, a.cumsum, a.P = _ptr(sig), _ptr(npts), _ptr(cums), P
        a.shs, a.sh_degree, a.M = _ptr(sh), int(sh_degree), M
        a.opacities = _ptr(opac)
        a.dL_dtriangle, a.dL_dsigma, a.dL_dopacity, a.dL_dsh = [_ptr(g) for g in grads]
        a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
        _set_cache(a, hit_cache, dev)
        vs = (_lib.TtView * len(rays))()
        keep = (verts, sig, npts, cums, sh, opac, bg, hit_cache)
        for i, ((ro, rd), (col, oth), (g, go)) in enumerate(zip(rays, forward_outputs, upstream)):
            ro, rd = _f32(ro, "ray_o", dev), _f32(rd, "ray_d", dev)
            col, oth = _f32(col, "colors", dev), _f32(oth, "others", dev)
            g, go = _f32(g, "dL_dpixels", dev), _f32(go, "dL_dothers", dev)
            vs[i].H, vs[i].W = int(ro.shape[0]), int(ro.shape[1])
            vs[i].ray_o, vs[i].ray_d = _ptr(ro), _ptr(rd)
            vs[i].colors, vs[i].others = _ptr(col), _ptr(oth)
            vs[i].dL_dpixels, vs[i].dL_dothers = _ptr(g), _ptr(go)
            keep = keep + (ro, rd, col, oth, g, go)
            keep = keep + self._interval_record(vs[i], vs[i].H, vs[i].W, intervals, None, i)
        check(self._h, lib.tt_backward_views(self._h, ctypes.byref(a), vs, len(rays), _stream()))
        self._keep = keep
        return grads

    def device_status(self):
        """Synchronises and raises if a bounded device loop gave up since the
        last check (no reference counterpart)."""
        check(self._h, lib.tt_device_status(self._h, _stream()))

    def _interval_record(self, view, H, W, intervals, records, i):
        keep = ()
        if intervals is not None and intervals[i] is not None:
            iv = _f32(intervals[i], "interval", self.device)
            if tuple(iv.shape) != (2, H, W):
                raise ValueError(f"interval of view {i} must be [2, {H}, {W}], got {tuple(iv.shape)}")
            view.interval = _ptr(iv)
            keep += (iv,)
        if records is not None and records[i] is not None:
            rec = records[i]
            if rec.dtype != torch.float32 or not rec.is_contiguous() or tuple(rec.shape) != (3, H, W):
                raise ValueError(f"record of view {i} must be a contiguous float32 [3, {H}, {W}] tensor")
            view.record = _ptr(rec)
            keep += (rec,)
        return keep

    def stats(self):
        """Synchronises; returns the handle's counters since reset_stats()."""
        s = _lib.TtStats()
        check(self._h, lib.tt_get_stats(self._h, ctypes.byref(s), _stream()))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def reset_stats(self):
        check(self._h, lib.tt_reset_stats(self._h, _stream()))

    def hit_stream(self, ray_o, ray_d, max_hits=64):
        """Test hook: first `max_hits` hits per ray ordered by (t, primitive)."""
        ro = _f32(ray_o, "ray_o", self.device).reshape(-1, 3)
        rd = _f32(ray_d, "ray_d", self.device).reshape(-1, 3)
        R = ro.shape[0]
        ids = torch.full((R, max_hits), -1, dtype=torch.int32, device=self.device)
        ts = torch.full((R, max_hits), float("inf"), dtype=torch.float32, device=self.device)
        counts = torch.zeros((R,), dtype=torch.int32, device=self.device)
        check(self._h, lib.tt_hit_stream(self._h, _ptr(ro), _ptr(rd), R, max_hits, _ptr(ids), _ptr(ts),
                                         _ptr(counts), _stream()))
        return ids, ts, counts
