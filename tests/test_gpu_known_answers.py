"""The CUDA path (through the C ABI) against the closed-form answers of
tests/known_answers.py, in every traversal configuration and both tmin
conventions: the window function and SH on an equilateral triangle, and a
stack of 60 sheets on one ray (chunked march with the closed interval's
repeated hit, near cut-off, 1/255 floor, 0.99 clamp, 1e-4 termination), with
the reference-semantics adjoint and the exact-adjoint forward's depth,
middepth and distortion. Images within 1e-5 relative (+1e-6), gradients
within 1e-5 relative (+1e-5)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import known_answers as ka  # noqa: E402
from diff_tritracer import _C  # noqa: E402
from gpu_helpers import gpu_backward, gpu_forward, settings  # noqa: E402
from test_oracle_known_answers import BG, close, expected_grads, upstream  # noqa: E402

CONFIGS = [("packets", 16, 0), ("packets", 32, 0), ("lanes", 16, 32), ("lanes", 16, 24)]
IDS = [f"{t}{k}s{s}" for t, k, s in CONFIGS]


def tracer(cfg, closed, exact_adjoint=False):
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=closed, exact_adjoint=exact_adjoint)
    tr.set_traversal(*cfg)
    return tr


@pytest.mark.parametrize("closed", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_window_function_sh_and_adjoint(cfg, closed):
    sc, ro, rd = ka.window_case()
    ans = ka.window_answers(sc, BG, closed)
    tr = tracer(cfg, closed)
    st = settings(bg=BG)
    f = gpu_forward(tr, sc, ro, rd, st)
    for i, a in enumerate(ans):
        close(f["color"][:, 0, i], a.color)
        close(f["others"][1:5, 0, i], np.concatenate([[1.0 - a.T], a.normal]))
        assert np.all(f["others"][[0, 5, 6], 0, i] == 0)
        if not a.blends:  # edge hits (Cx = 0) and misses
            close(f["color"][:, 0, i], BG.astype(np.float32), rtol=0, atol=0)
    close(f["max_blending"][0], max(a.blends[0].alpha for a in ans if a.blends))
    assert f["density"][0] == 1
    g, go = upstream(ro.shape[1], seed=4)
    b = gpu_backward(tr, sc, ro, rd, st, f["color"], f["others"], g, go)
    tr.device_status()
    dop, dsig, dsh = expected_grads(ans, sc, g, go)
    close(b["dopac"], dop, atol=1e-5)
    close(b["dsigma"], dsig, atol=1e-5)
    close(b["dsh"], dsh, atol=1e-5)


@pytest.mark.parametrize("closed", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("z0", [3.0, -0.225], ids=["above", "inside"])
@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_stack_of_sheets(cfg, z0, closed):
    sc, zs = ka.stack_case()
    a = ka.stack_answer(sc, zs, z0, BG, closed)
    ro, rd = ka.rays([(0.0, 0.0)], z0)
    tr = tracer(cfg, closed)
    st = settings(bg=BG)
    f = gpu_forward(tr, sc, ro, rd, st)
    close(f["color"][:, 0, 0], a.color)
    close(f["others"][1:5, 0, 0], np.concatenate([[1.0 - a.T], a.normal]))
    blended = sorted({b.prim for b in a.blends})
    want_maxb, want_density, want_scaling = np.zeros(sc.P), np.zeros(sc.P), np.zeros(sc.P)
    for b in a.blends:
        want_maxb[b.prim] = max(want_maxb[b.prim], b.alpha * b.T)
    want_density[blended] = 1
    for p in blended:
        want_scaling[p] = ka.scaling_of(z0, float(zs[p]))
    close(f["max_blending"], want_maxb)
    np.testing.assert_array_equal(f["density"], want_density)
    close(f["scaling"], want_scaling)
    g, go = upstream(1, seed=5)
    b = gpu_backward(tr, sc, ro, rd, st, f["color"], f["others"], g, go)
    tr.device_status()
    dop, dsig, dsh = expected_grads([a], sc, g, go)
    close(b["dopac"], dop, atol=1e-5)
    close(b["dsigma"], dsig, atol=1e-5)
    close(b["dsh"], dsh, atol=1e-5)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_stack_exact_forward_outputs(cfg):
    sc, zs = ka.stack_case()
    a = ka.stack_answer(sc, zs, 3.0, BG, True)
    ro, rd = ka.rays([(0.0, 0.0)], 3.0)
    tr = tracer(cfg, True, exact_adjoint=True)
    f = gpu_forward(tr, sc, ro, rd, settings(bg=BG))
    tr.device_status()
    close(f["others"][0, 0, 0], a.depth)
    close(f["others"][5, 0, 0], a.middepth)
    close(f["others"][6, 0, 0], a.distortion)
    close(f["color"][:, 0, 0], a.color)
