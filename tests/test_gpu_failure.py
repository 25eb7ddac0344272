"""Failure detection on the GPU without a fault: a bounded device loop runs
out on real input, the kernel ends the ray and records the reason, the host
reads it with tt_device_status (TT_ERR_TIMEOUT -> TracerError), and the
handle keeps working.

The input: 20 coincident copies of one triangle with opacity below the 1/255
floor. Under the closed interval [last_hit_t, 1000] the reference's march
re-traces from their common t and gets the same 16 hits back, all skipped,
forever (tritracer/forward.cu:161-215 has no bound). Here each chunk boundary
that makes no progress is counted; past 16 the ray ends with the timeout
status. The open interval steps past the common t and finishes cleanly."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import known_answers as ka  # noqa: E402
from diff_tritracer import _C, _lib  # noqa: E402
from gpu_helpers import gpu_forward, settings  # noqa: E402
from test_gpu_known_answers import CONFIGS, IDS  # noqa: E402

BG = np.array([0.25, 0.5, 0.75], np.float32)


def coincident(n=20, opacity=1e-3):
    return ka.scene([0.0] * n, [opacity] * n, [1.0] * n, np.zeros((n, 16, 3)), 3)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_no_progress_march_reports_timeout_and_handle_recovers(cfg):
    sc = coincident()
    ro, rd = ka.rays([(0.0, 0.0), (0.1, 0.05), (2.0, 0.0)], 3.0)  # two rays through the stack, one miss
    closed = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=True)
    closed.set_traversal(*cfg)
    out = gpu_forward(closed, sc, ro, rd, settings(bg=BG))
    with pytest.raises(_lib.TracerError, match="bounded device loop") as err:
        closed.device_status()
    assert err.value.code == _lib.TT_ERR_TIMEOUT
    np.testing.assert_array_equal(out["color"][:, 0, :], np.repeat(BG[:, None], 3, 1))  # every hit was skipped
    # the status was cleared and the handle still traces
    stack, zs = ka.stack_case()
    a = ka.stack_answer(stack, zs, 3.0, BG, True)
    out = gpu_forward(closed, stack, *ka.rays([(0.0, 0.0)], 3.0), settings(bg=BG))
    closed.device_status()
    np.testing.assert_allclose(out["color"][:, 0, 0], a.color, rtol=1e-5, atol=1e-6)
    # the open interval moves past the common t
    open_ = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=False)
    open_.set_traversal(*cfg)
    out = gpu_forward(open_, sc, ro, rd, settings(bg=BG))
    open_.device_status()
    np.testing.assert_array_equal(out["color"][:, 0, :], np.repeat(BG[:, None], 3, 1))


def test_visible_coincident_hits_terminate_without_error():
    """The same stack at opacity 0.5: the closed interval composites the
    repeated hits until T < 1e-4 ends the ray well before the bound."""
    sc = coincident(opacity=0.5)
    ro, rd = ka.rays([(0.0, 0.0)], 3.0)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", tmin_inclusive=True)
    out = gpu_forward(tr, sc, ro, rd, settings(bg=BG))
    tr.device_status()
    assert out["others"][1, 0, 0] > 1 - 2e-4
