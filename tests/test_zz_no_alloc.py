"""tt_forward_noalloc: the forward trace for callers that cannot allocate device
memory (an engine plugin that only receives each call's input and output
buffers, a frame loop with a fixed memory budget). It builds the BVH and runs
the trace out of one fixed file-scope device array instead of cudaMalloc'd
memory, for at most TT_NOALLOC_MAX_TRIANGLES triangles.

Called here through the C ABI with ctypes and checked three ways:
* against the allocating tt_forward on the same inputs, within the forward
  tolerance of the parity tests, at 0, 1, 4000 and the maximum 8192
  triangles, under both tmin conventions;
* against the FP64 oracle directly, as the parity tests check tt_forward;
* calls in a row on different scenes (the array keeps the previous call's
  contents: a stale BVH, flag or counter would show), with the device's free
  memory and the torch allocator's counters unchanged across each call.
tt_noalloc_status reports a bounded loop that gave up (the coincident-triangle
input of the failure test) and clears itself.

This file is collected last on purpose and must also pass alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import known_answers as ka  # noqa: E402
from diff_tritracer import _C, _lib  # noqa: E402
from gpu_helpers import MARGIN, flagged_prims  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

RTOL, ATOL = 1e-5, 1e-6
MAX_TRIANGLES = 8192  # TT_NOALLOC_MAX_TRIANGLES in include/tritracer.h
TT_ERR_TOO_LARGE = 7

lib = _lib.lib
lib.tt_forward_noalloc.argtypes = [ctypes.POINTER(_lib.TtConfig), ctypes.POINTER(_lib.TtFwdArgs), ctypes.c_void_p]
lib.tt_forward_noalloc.restype = ctypes.c_int
lib.tt_noalloc_status.argtypes = [ctypes.c_void_p]
lib.tt_noalloc_status.restype = ctypes.c_int

DEV = torch.device("cuda:0")
BG = np.array([0.05, 0.1, 0.2], np.float32)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def p(t):
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class NoallocCall:
    """Device inputs, outputs and the argument block of one call, all made
    before the call so that the call itself is the only thing measured."""

    def __init__(self, sc, ro, rd, bg=BG, tmin_inclusive=1):
        H, W = ro.shape[:2]
        P = sc.P
        self.keep = dict(ro=T(ro), rd=T(rd), verts=T(sc.verts), npts=T(sc.num_points), cums=T(sc.cumsum),
                         shs=T(sc.shs), opac=T(sc.opacities), sigma=T(sc.sigma), bg=T(bg))
        self.out = dict(color=torch.full((3, H, W), -1.0, device=DEV), others=torch.full((7, H, W), -1.0, device=DEV),
                        max_blending=torch.full((max(P, 1),), -1.0, device=DEV),
                        scaling=torch.zeros(max(P, 1), device=DEV), density=torch.zeros(max(P, 1), device=DEV))
        k, o = self.keep, self.out
        a = _lib.TtFwdArgs()
        a.H, a.W = H, W
        a.ray_o, a.ray_d = p(k["ro"]), p(k["rd"])
        a.vertices, a.num_vertices = p(k["verts"]), k["verts"].numel() // 3
        a.num_points, a.cumsum, a.P = p(k["npts"]), p(k["cums"]), P
        a.shs, a.sh_degree, a.M = p(k["shs"]), sc.sh_degree, sc.shs.shape[1]
        a.colors_precomp = ctypes.c_void_p(0)
        a.opacities, a.sigma = p(k["opac"]), p(k["sigma"])
        a.scaling, a.density_factor = p(o["scaling"]), p(o["density"])
        a.bg, a.extra, a.extra_len = p(k["bg"]), ctypes.c_void_p(0), 0
        a.rebuild_gas, a.debug = 0, 0
        a.out_color, a.out_others, a.max_blending = p(o["color"]), p(o["others"]), p(o["max_blending"])
        a.gpu_time_ms = ctypes.cast(None, ctypes.POINTER(ctypes.c_float))
        self.args = a
        self.cfg = _lib.TtConfig()
        self.cfg.variant, self.cfg.tmin_inclusive = 0, tmin_inclusive
        self.P = P
        torch.cuda.synchronize()

    def run(self):
        rc = lib.tt_forward_noalloc(ctypes.byref(self.cfg), ctypes.byref(self.args), stream())
        torch.cuda.synchronize()
        return rc

    def result(self):
        P = self.P
        r = {k: v.cpu().numpy() for k, v in self.out.items()}
        for k in ("max_blending", "scaling", "density"):
            r[k] = r[k][:P]
        return r


def allocating_forward(sc, ro, rd, bg=BG, tmin_inclusive=True):
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=tmin_inclusive)
    P = sc.P
    res = tr.trace_forward(T(ro), T(rd), T(sc.verts), T(sc.sigma), T(sc.num_points), T(sc.cumsum), P, T(sc.shs),
                           sc.sh_degree, torch.empty(0, device=DEV), T(sc.opacities), torch.zeros(P, device=DEV),
                           torch.zeros(P, device=DEV), T(bg), torch.zeros(5, device=DEV), 0, False).data
    torch.cuda.synchronize()
    tr.device_status()
    color, others, _, scaling, density, maxb = res
    return {k: v.cpu().numpy() for k, v in dict(color=color, others=others, scaling=scaling, density=density,
                                                 max_blending=maxb).items()}


def assert_same(got, want, what):
    for key in ("color", "others", "max_blending", "scaling", "density"):
        np.testing.assert_allclose(got[key], want[key], rtol=RTOL, atol=ATOL, err_msg=f"{what}: {key}")


def scene_of(P, seed):
    if P == 0:
        sc = dense_scene(seed=seed, P=1)
        sc.verts, sc.num_points, sc.cumsum = sc.verts[:0], sc.num_points[:0], sc.cumsum[:0]
        sc.opacities, sc.sigma, sc.shs = sc.opacities[:0], sc.sigma[:0], sc.shs[:0]
        return sc
    if P == 1:  # one large triangle facing the camera, so the rays do hit it
        return ka.scene([0.0], [0.8], [1.0], np.full((1, 16, 3), 0.2), 3)
    return dense_scene(seed=seed, P=P)


def device_memory_state():
    free, _ = torch.cuda.mem_get_info(DEV)
    st = torch.cuda.memory_stats(DEV)
    return free, st.get("allocation.all.allocated", 0), st.get("segment.all.allocated", 0)


@pytest.mark.parametrize("incl", [1, 0], ids=["closed", "open"])
@pytest.mark.parametrize("P", [0, 1, 4000, MAX_TRIANGLES])
def test_noalloc_matches_allocating_forward(P, incl):
    sc = scene_of(P, seed=7)
    ro, rd = dense_view(H=48, W=64)
    want = allocating_forward(sc, ro, rd, tmin_inclusive=bool(incl))
    call = NoallocCall(sc, ro, rd, tmin_inclusive=incl)
    assert call.run() == 0
    assert lib.tt_noalloc_status(stream()) == 0
    got = call.result()
    assert_same(got, want, f"P={P}")
    if P == 0:
        np.testing.assert_array_equal(got["color"], np.broadcast_to(BG[:, None, None], got["color"].shape))
    elif P == 1:
        assert (got["others"][1] > 0).sum() > 10  # some rays blended the triangle
    else:
        assert want["color"].mean() > 0.05


def test_noalloc_vs_fp64_oracle(oracle):
    sc = dense_scene(seed=7, P=4000)
    ro, rd = dense_view(H=48, W=64)
    H, W = ro.shape[:2]
    call = NoallocCall(sc, ro, rd)
    assert call.run() == 0
    assert lib.tt_noalloc_status(stream()) == 0
    out = call.result()
    ref = oracle.forward(sc, ro, rd, bg=BG, precision=64, exact=True, canonical=True, tmin_inclusive=True,
                         record=256, nthreads=8)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.mean() > 0.97, ok.mean()
    for key in ("color", "others"):
        a, b = out[key][:, ok], getattr(ref, key)[:, ok]
        assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + ATOL), key
    skip = np.zeros(sc.P, bool)
    skip[flagged_prims(ref, H, W, ok)] = True
    np.testing.assert_array_equal(out["density"][~skip], ref.density[~skip])
    np.testing.assert_allclose(out["max_blending"][~skip], ref.max_blending[~skip], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(out["scaling"][~skip], ref.scaling[~skip], rtol=1e-6, atol=1e-9)


def test_calls_in_a_row_on_different_scenes_allocate_nothing():
    ro, rd = dense_view(H=48, W=64)
    scenes = [dense_scene(seed=7, P=4000), dense_scene(seed=21, P=1500), dense_scene(seed=7, P=4000)]
    wants = [allocating_forward(sc, ro, rd) for sc in scenes]
    calls = [NoallocCall(sc, ro, rd) for sc in scenes]
    assert calls[0].run() == 0  # the first call on the device may load the module and its array
    for i, (call, want) in enumerate(zip(calls, wants)):
        before = device_memory_state()
        assert call.run() == 0
        after = device_memory_state()
        # no allocation: the device's free memory did not shrink (the driver
        # may release memory of its own meanwhile) and the torch allocator
        # made no allocation and reserved no segment
        assert after[0] >= before[0] and after[1:] == before[1:], (i, before, after)
        assert lib.tt_noalloc_status(stream()) == 0
        assert_same(call.result(), want, f"call {i}")
    # the smaller scene really differs from the others
    assert np.abs(wants[1]["color"] - wants[0]["color"]).max() > 1e-2


def test_noalloc_status_reports_a_bound_that_ran_out():
    sc = ka.scene([0.0] * 20, [1e-3] * 20, [1.0] * 20, np.zeros((20, 16, 3)), 3)  # coincident, below 1/255
    ro, rd = ka.rays([(0.0, 0.0), (0.1, 0.05), (2.0, 0.0)], 3.0)
    call = NoallocCall(sc, ro, rd, bg=np.array([0.25, 0.5, 0.75], np.float32), tmin_inclusive=1)
    assert call.run() == 0
    assert lib.tt_noalloc_status(stream()) == _lib.TT_ERR_TIMEOUT
    assert lib.tt_noalloc_status(stream()) == 0  # cleared
    # the open interval steps past the common t
    call = NoallocCall(sc, ro, rd, bg=np.array([0.25, 0.5, 0.75], np.float32), tmin_inclusive=0)
    assert call.run() == 0
    assert lib.tt_noalloc_status(stream()) == 0


def test_noalloc_rejects_scenes_beyond_capacity():
    sc = dense_scene(seed=7, P=MAX_TRIANGLES + 1)
    ro, rd = dense_view(H=8, W=8)
    call = NoallocCall(sc, ro, rd)
    assert call.run() == TT_ERR_TOO_LARGE
    assert np.all(call.result()["color"] == -1.0)  # nothing was enqueued
