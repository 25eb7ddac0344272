"""The index-checked debug build (`make bounds`: libtritracer_bounds.so,
-DTT_BOUNDS_CHECK). compute-sanitizer is not available on these GPUs, so the
kernels check their own node, leaf, warp-stack and primitive indices; a
failed check records TT_ERR_BOUNDS (read by tt_device_status) and skips the
access. The GPU parity suites run here against that build in a subprocess
(TRITRACER_LIB): every test calls device_status after its launches, so any
violation fails it."""
import os
import subprocess
import sys

import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "diff-triangle-tracer_b200", "diff_tritracer", "libtritracer_bounds.so")
SUITES = ["test_gpu_parity.py", "test_gpu_known_answers.py", "test_gpu_hit_cache.py", "test_gpu_batch.py",
          "test_gpu_secondary.py", "test_gpu_edge_cases.py", "test_gpu_failure.py"]


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_parity_suites_pass_under_index_checks():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} is missing: build it with `make -C diff-triangle-tracer_b200 bounds`")
    env = dict(os.environ, TRITRACER_LIB=LIB)
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"]
    cmd += [os.path.join(ROOT, "tests", s) for s in SUITES]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-2000:]
    assert "passed" in res.stdout


def test_library_override_is_loaded():
    code = "from diff_tritracer import _lib; print(_lib.LIB_PATH)"
    env = dict(os.environ, TRITRACER_LIB=LIB, PYTHONPATH=os.path.join(ROOT, "diff-triangle-tracer_b200"))
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    if not os.path.exists(LIB):
        pytest.skip("index-checked build not present")
    assert out.returncode == 0 and out.stdout.strip() == LIB, out.stderr[-1000:]
