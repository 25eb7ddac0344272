"""tt_forward_noalloc: the forward trace for callers that cannot allocate device
memory (an engine plugin that only receives each call's input and output
buffers, a frame loop with a fixed memory budget). It builds the BVH and runs
the trace out of one fixed file-scope device array instead of cudaMalloc'd
memory, for at most TT_NOALLOC_MAX_TRIANGLES triangles.

Called here through the C ABI with ctypes, twice in a row (the array keeps the
previous call's contents, so the second call checks that each call clears
what must start at zero), and compared with the allocating tt_forward on the
same inputs, within the forward tolerance of the parity tests. This file is
collected last on purpose and must also pass alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, _lib  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL = 1e-5, 1e-6
MAX_TRIANGLES = 8192  # TT_NOALLOC_MAX_TRIANGLES in include/tritracer.h
TT_ERR_TOO_LARGE = 7

lib = _lib.lib
lib.tt_forward_noalloc.argtypes = [ctypes.POINTER(_lib.TtConfig), ctypes.POINTER(_lib.TtFwdArgs), ctypes.c_void_p]
lib.tt_forward_noalloc.restype = ctypes.c_int

DEV = torch.device("cuda:0")


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def p(t):
    return ctypes.c_void_p(t.data_ptr())


def noalloc_forward(sc, ro, rd, bg, P=None):
    P = sc.P if P is None else P
    H, W = ro.shape[:2]
    keep = dict(ro=T(ro), rd=T(rd), verts=T(sc.verts), npts=T(sc.num_points), cums=T(sc.cumsum), shs=T(sc.shs),
                opac=T(sc.opacities), sigma=T(sc.sigma), bg=T(bg))
    out = dict(color=torch.full((3, H, W), -1.0, device=DEV), others=torch.full((7, H, W), -1.0, device=DEV),
               max_blending=torch.full((sc.P,), -1.0, device=DEV), scaling=torch.zeros(sc.P, device=DEV),
               density=torch.zeros(sc.P, device=DEV))
    a = _lib.TtFwdArgs()
    a.H, a.W = H, W
    a.ray_o, a.ray_d = p(keep["ro"]), p(keep["rd"])
    a.vertices, a.num_vertices = p(keep["verts"]), keep["verts"].numel() // 3
    a.num_points, a.cumsum, a.P = p(keep["npts"]), p(keep["cums"]), P
    a.shs, a.sh_degree, a.M = p(keep["shs"]), sc.sh_degree, sc.shs.shape[1]
    a.colors_precomp = ctypes.c_void_p(0)
    a.opacities, a.sigma = p(keep["opac"]), p(keep["sigma"])
    a.scaling, a.density_factor = p(out["scaling"]), p(out["density"])
    a.bg, a.extra, a.extra_len = p(keep["bg"]), ctypes.c_void_p(0), 0
    a.rebuild_gas, a.debug = 0, 0
    a.out_color, a.out_others, a.max_blending = p(out["color"]), p(out["others"]), p(out["max_blending"])
    a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
    cfg = _lib.TtConfig()
    cfg.variant, cfg.tmin_inclusive = 0, 1
    rc = lib.tt_forward_noalloc(ctypes.byref(cfg), ctypes.byref(a),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, {k: v.cpu().numpy() for k, v in out.items()}


def allocating_forward(sc, ro, rd, bg):
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx")
    P = sc.P
    res = tr.trace_forward(T(ro), T(rd), T(sc.verts), T(sc.sigma), T(sc.num_points), T(sc.cumsum), P, T(sc.shs),
                           sc.sh_degree, torch.empty(0, device=DEV), T(sc.opacities), torch.zeros(P, device=DEV),
                           torch.zeros(P, device=DEV), T(bg), torch.zeros(5, device=DEV), 0, False).data
    torch.cuda.synchronize()
    color, others, _, scaling, density, maxb = res
    return {k: v.cpu().numpy() for k, v in dict(color=color, others=others, scaling=scaling, density=density,
                                                 max_blending=maxb).items()}


def test_noalloc_forward_matches_allocating_forward_twice():
    sc = dense_scene(seed=7, P=4000)
    ro, rd = dense_view(H=48, W=64)
    bg = np.array([0.05, 0.1, 0.2], np.float32)
    want = allocating_forward(sc, ro, rd, bg)
    assert want["color"].mean() > 0.05
    for call in range(2):
        rc, got = noalloc_forward(sc, ro, rd, bg)
        assert rc == 0, (call, rc)
        for key in ("color", "others", "max_blending", "scaling", "density"):
            np.testing.assert_allclose(got[key], want[key], rtol=RTOL, atol=ATOL, err_msg=f"call {call}: {key}")


def test_noalloc_rejects_scenes_beyond_capacity():
    sc = dense_scene(seed=7, P=MAX_TRIANGLES + 1)
    ro, rd = dense_view(H=8, W=8)
    rc, got = noalloc_forward(sc, ro, rd, np.zeros(3, np.float32))
    assert rc == TT_ERR_TOO_LARGE
    assert np.all(got["color"] == -1.0)  # nothing was enqueued
