"""Test infrastructure (oracle): ctypes bindings for the CPU restatement
(_lib/liboracle.so) and for the host build of the reference's own device
sources (_ref/libtritracer_ref.so). Only tests, the smoke check and the
benchmark's CPU baseline leg import this module.

Both libraries are built by ``make -C oracle`` (``__graft_entry__.build()``
runs it); the reference build needs the reference's sources and is skipped
where they are absent.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libtritracer_ref.so")

_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


class OrArgs(ctypes.Structure):
    _fields_ = [
        ("H", ctypes.c_int), ("W", ctypes.c_int),
        ("ray_o", _fp), ("ray_d", _fp), ("verts", _fp),
        ("num_points", _ip), ("cumsum", _ip), ("P", ctypes.c_int),
        ("shs", _fp), ("sh_degree", ctypes.c_int), ("M", ctypes.c_int),
        ("opacities", _fp), ("sigma", _fp), ("bg", _fp),
        ("extra", _fp), ("extra_len", ctypes.c_int),
        ("variant", ctypes.c_int), ("tmin_inclusive", ctypes.c_int),
        ("canonical_ties", ctypes.c_int), ("exact_geometry", ctypes.c_int),
        ("nthreads", ctypes.c_int), ("row_begin", ctypes.c_int), ("row_end", ctypes.c_int),
        ("colors", ctypes.c_void_p), ("others", ctypes.c_void_p),
        ("dL_dpixels", _fp), ("dL_dothers", _fp),
        ("max_rec", ctypes.c_int), ("rec_ids", _ip), ("rec_count", _ip), ("margin", _fp),
        ("interval", _fp),
        ("material", _ip), ("ior", _fp), ("env", _fp), ("env_h", ctypes.c_int), ("env_w", ctypes.c_int),
        ("max_depth", ctypes.c_int), ("exact_adjoint", ctypes.c_int),
        ("precomp", _fp), ("dprecomp", ctypes.c_void_p),
        ("max_chunks", ctypes.c_int), ("chunk_ids", ctypes.POINTER(ctypes.c_uint32)), ("chunk_tmin", _fp),
        ("chunk_count", _ip),
        ("denv", ctypes.c_void_p), ("dior", ctypes.c_void_p), ("ior_fresnel", _fp),
    ]


def _ptr(a, t=_fp):
    if a is None:
        return ctypes.cast(None, t)
    return a.ctypes.data_as(t)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


@dataclass
class FwdResult:
    color: np.ndarray
    others: np.ndarray
    scaling: np.ndarray
    density: np.ndarray
    max_blending: np.ndarray
    rec_ids: np.ndarray | None = None
    rec_count: np.ndarray | None = None
    margin: np.ndarray | None = None
    chunk_ids: np.ndarray | None = None  # [H*W, chunks, 16] (reference only, `chunks` > 0)
    chunk_tmin: np.ndarray | None = None  # [H*W, chunks]
    chunk_count: np.ndarray | None = None  # [H*W]


@dataclass
class BwdResult:
    dtri: np.ndarray
    dsigma: np.ndarray
    dopac: np.ndarray
    dsh: np.ndarray
    dcolors: np.ndarray | None = None
    denv: np.ndarray | None = None  # secondary rays: [env_h, env_w, 3]
    dior: np.ndarray | None = None  # secondary rays: [P]


class _Runner:
    """One of the two CPU implementations: the restatement ("or_") or the
    reference's own code ("ref_")."""

    def __init__(self, path: str, prefix: str):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        L = self.lib
        getattr(L, prefix + "_scene_new").restype = ctypes.c_void_p
        getattr(L, prefix + "_scene_new").argtypes = [_fp, _ip, ctypes.c_int]
        getattr(L, prefix + "_scene_free").argtypes = [ctypes.c_void_p]
        self._scenes = {}

    def _scene(self, scene):
        key = id(scene)
        ent = self._scenes.get(key)
        if ent is None or ent[0] is not scene:
            verts = _c(scene.verts, np.float32)
            cumsum = _c(scene.cumsum, np.int32)
            h = getattr(self.lib, self.prefix + "_scene_new")(_ptr(verts), _ptr(cumsum, _ip), scene.P)
            ent = (scene, h, verts, cumsum)
            self._scenes[key] = ent
        return ent

    def _args(self, scene, ray_o, ray_d, bg, extra, variant, tmin_inclusive, canonical, exact, nthreads, rows):
        sc, _, verts, cumsum = self._scene(scene)
        H, W = ray_o.shape[0], ray_o.shape[1]
        keep = dict(
            ray_o=_c(ray_o, np.float32), ray_d=_c(ray_d, np.float32), verts=verts, cumsum=cumsum,
            num_points=_c(scene.num_points, np.int32), shs=_c(scene.shs, np.float32),
            opac=_c(scene.opacities, np.float32), sigma=_c(scene.sigma, np.float32),
            bg=_c(bg if bg is not None else np.zeros(3), np.float32),
            extra=_c(extra if extra is not None else np.zeros(5), np.float32),
        )
        a = OrArgs()
        a.H, a.W = H, W
        a.ray_o, a.ray_d = _ptr(keep["ray_o"]), _ptr(keep["ray_d"])
        a.verts, a.num_points, a.cumsum = _ptr(verts), _ptr(keep["num_points"], _ip), _ptr(cumsum, _ip)
        a.P = scene.P
        a.shs, a.sh_degree, a.M = _ptr(keep["shs"]), scene.sh_degree, scene.shs.shape[1]
        a.opacities, a.sigma, a.bg = _ptr(keep["opac"]), _ptr(keep["sigma"]), _ptr(keep["bg"])
        a.extra, a.extra_len = _ptr(keep["extra"]), keep["extra"].size
        a.variant, a.tmin_inclusive = variant, int(tmin_inclusive)
        a.canonical_ties, a.exact_geometry = int(canonical), int(exact)
        a.nthreads = nthreads
        a.row_begin, a.row_end = (rows if rows is not None else (0, 0))
        return a, keep

    @staticmethod
    def _interval(a, keep, interval):
        """Optional proposed interval per ray, [2, H, W] (t_near, t_far)."""
        if interval is None:
            return
        keep["interval"] = _c(interval, np.float32)
        if keep["interval"].shape != (2, a.H, a.W):
            raise ValueError("interval must be [2, H, W]")
        a.interval = _ptr(keep["interval"])

    @staticmethod
    def _secondary(a, keep, secondary):
        """Secondary-ray inputs: dict(material [P] int, ior [P], env [h, w, 3],
        max_depth; optional ior_fresnel [P]: the IOR of the Fresnel share
        only, for finite differences of the IOR gradient)."""
        if secondary is None:
            return ""
        keep["material"] = _c(secondary["material"], np.int32)
        keep["ior"] = _c(secondary["ior"], np.float32)
        keep["env"] = _c(secondary["env"], np.float32)
        a.material, a.ior, a.env = _ptr(keep["material"], _ip), _ptr(keep["ior"]), _ptr(keep["env"])
        a.env_h, a.env_w = keep["env"].shape[0], keep["env"].shape[1]
        a.max_depth = int(secondary.get("max_depth", 2))
        if secondary.get("ior_fresnel") is not None:
            keep["ior_fresnel"] = _c(secondary["ior_fresnel"], np.float32)
            a.ior_fresnel = _ptr(keep["ior_fresnel"])
        return "secondary_"

    def forward(self, scene, ray_o, ray_d, bg=None, extra=None, variant=0, precision=32, tmin_inclusive=True,
                canonical=False, exact=False, nthreads=1, scaling=None, density=None, record=0, rows=None,
                interval=None, secondary=None, exact_adjoint=False, precomp=None, chunks=0):
        """`chunks` > 0 (the reference's own code only): also log, per ray, up
        to that many of its k-closest queries (lower bound and the 16 ids the
        any-hit program kept)."""
        a, keep = self._args(scene, ray_o, ray_d, bg, extra, variant, tmin_inclusive, canonical, exact, nthreads, rows)
        a.exact_adjoint = int(exact_adjoint)
        if precomp is not None:
            keep["precomp"] = _c(precomp, np.float32)
            a.precomp = _ptr(keep["precomp"])
        self._interval(a, keep, interval)
        sec = self._secondary(a, keep, secondary)
        dt = np.float32 if precision == 32 else np.float64
        H, W, P = a.H, a.W, scene.P
        scaling = np.zeros(P, dt) if scaling is None else _c(scaling, dt).reshape(-1).copy()
        density = np.zeros(P, dt) if density is None else _c(density, dt).reshape(-1).copy()
        color = np.zeros((3, H, W), dt)
        others = np.zeros((7, H, W), dt)
        maxb = np.zeros(P, dt)
        rec_ids = rec_count = margin = None
        if record:
            rec_ids = np.full((H * W, record), -1, np.int32)
            rec_count = np.zeros(H * W, np.int32)
            margin = np.zeros(H * W, np.float32)
            a.max_rec, a.rec_ids, a.rec_count, a.margin = record, _ptr(rec_ids, _ip), _ptr(rec_count, _ip), _ptr(margin)
        chunk_ids = chunk_tmin = chunk_count = None
        if chunks:
            assert self.prefix == "ref", "the query log is a hook of the reference's host build"
            chunk_ids = np.full((H * W, chunks, 16), 0xFFFFFFFF, np.uint32)
            chunk_tmin = np.full((H * W, chunks), np.nan, np.float32)
            chunk_count = np.zeros(H * W, np.int32)
            a.max_chunks = chunks
            a.chunk_ids = _ptr(chunk_ids, ctypes.POINTER(ctypes.c_uint32))
            a.chunk_tmin, a.chunk_count = _ptr(chunk_tmin), _ptr(chunk_count, _ip)
        t = ctypes.POINTER(ctypes.c_float if precision == 32 else ctypes.c_double)
        if self.prefix == "ref":
            assert precision == 32
            fn = self.lib.ref_forward
        else:
            fn = getattr(self.lib, f"or_forward_{sec}f{precision}")
        fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(OrArgs)] + [t] * 5
        rc = fn(self._scene(scene)[1], ctypes.byref(a), _ptr(scaling, t), _ptr(density, t), _ptr(color, t),
                _ptr(others, t), _ptr(maxb, t))
        if rc != 0:
            raise RuntimeError(f"{self.prefix} forward failed ({rc})")
        return FwdResult(color, others, scaling, density, maxb, rec_ids, rec_count, margin, chunk_ids, chunk_tmin,
                         chunk_count)

    def backward(self, scene, ray_o, ray_d, colors, others, dL_dpixels, dL_dothers, bg=None, precision=32,
                 tmin_inclusive=True, canonical=False, exact=False, nthreads=1, rows=None, interval=None,
                 secondary=None, exact_adjoint=False, precomp=None):
        a, keep = self._args(scene, ray_o, ray_d, bg, None, 0, tmin_inclusive, canonical, exact, nthreads, rows)
        a.exact_adjoint = int(exact_adjoint)
        dcolors = None
        if precomp is not None:
            keep["precomp"] = _c(precomp, np.float32)
            a.precomp = _ptr(keep["precomp"])
            dcolors = np.zeros((scene.P, 3), np.float32 if precision == 32 else np.float64)
            a.dprecomp = dcolors.ctypes.data
        self._interval(a, keep, interval)
        sec = self._secondary(a, keep, secondary)
        dt = np.float32 if precision == 32 else np.float64
        keep["colors"] = _c(colors, dt)
        keep["others"] = _c(others, dt)
        keep["g"] = _c(dL_dpixels, np.float32)
        keep["go"] = _c(dL_dothers, np.float32)
        a.colors = keep["colors"].ctypes.data
        a.others = keep["others"].ctypes.data
        a.dL_dpixels, a.dL_dothers = _ptr(keep["g"]), _ptr(keep["go"])
        P, M = scene.P, scene.shs.shape[1]
        npts = int(scene.num_points[-1] + scene.cumsum[-1]) if P else 0
        dtri = np.zeros((npts, 3), dt)
        dsigma = np.zeros(P, dt)
        dopac = np.zeros(P, dt)
        dsh = np.zeros((P, M, 3), dt)
        denv = dior = None
        if sec:
            denv = np.zeros(keep["env"].shape, dt)
            dior = np.zeros(P, dt)
            a.denv, a.dior = denv.ctypes.data, dior.ctypes.data
        t = ctypes.POINTER(ctypes.c_float if precision == 32 else ctypes.c_double)
        if self.prefix == "ref":
            assert precision == 32
            fn = self.lib.ref_backward
        else:
            fn = getattr(self.lib, f"or_backward_{sec}f{precision}")
        fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(OrArgs)] + [t] * 4
        rc = fn(self._scene(scene)[1], ctypes.byref(a), _ptr(dtri, t), _ptr(dsigma, t), _ptr(dopac, t), _ptr(dsh, t))
        if rc != 0:
            raise RuntimeError(f"{self.prefix} backward failed ({rc})")
        res = BwdResult(dtri, dsigma, dopac, dsh)
        res.dcolors = dcolors
        res.denv, res.dior = denv, dior
        return res

    def close(self):
        for _, h, _, _ in self._scenes.values():
            getattr(self.lib, self.prefix + "_scene_free")(h)
        self._scenes.clear()


class Oracle(_Runner):
    def __init__(self, path: str = LIB_PATH):
        super().__init__(path, "or")

    def hit_stream(self, scene, ray_o, ray_d, max_hits=64, tmax=1000.0, nthreads=1):
        """All hits in [0, tmax] per ray, ordered by (t, id): (ids, ts, counts)."""
        ro = _c(ray_o, np.float32).reshape(-1, 3)
        rd = _c(ray_d, np.float32).reshape(-1, 3)
        R = ro.shape[0]
        ids = np.full((R, max_hits), 0xFFFFFFFF, np.uint32)
        ts = np.full((R, max_hits), np.inf, np.float32)
        counts = np.zeros(R, np.int32)
        fn = self.lib.or_hit_stream
        fn.argtypes = [ctypes.c_void_p, _fp, _fp, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                       ctypes.POINTER(ctypes.c_uint32), _fp, _ip, ctypes.c_int]
        fn(self._scene(scene)[1], _ptr(ro), _ptr(rd), R, tmax, max_hits, _ptr(ids, ctypes.POINTER(ctypes.c_uint32)),
           _ptr(ts), _ptr(counts, _ip), nthreads)
        return ids, ts, counts

    def isect(self, o, d, v0, v1, v2):
        t = ctypes.c_float(0)
        fn = self.lib.or_isect
        fn.argtypes = [_fp] * 5 + [_fp]
        arrs = [_c(x, np.float32) for x in (o, d, v0, v1, v2)]
        hit = fn(*[_ptr(x) for x in arrs], ctypes.byref(t))
        return bool(hit), t.value


class Reference(_Runner):
    def __init__(self, path: str = REF_PATH):
        super().__init__(path, "ref")


def oracle_available() -> bool:
    return os.path.exists(LIB_PATH)


def reference_available() -> bool:
    return os.path.exists(REF_PATH)
