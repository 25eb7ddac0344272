"""The reference's debug snapshot (diff_tritracer/__init__.py:96-107,
:183-194 there): with `debug` on, a call that raises leaves CPU copies of its
arguments in snapshot_fw.dump / snapshot_bw.dump before the error
propagates; with `debug` off nothing is written. The helper is checked on
the CPU; the forward's use of it through `Tracer` on the GPU."""
import os

import numpy as np
import pytest
import torch

import diff_tritracer


def test_snapshot_written_only_with_debug_and_on_error(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    args = (torch.arange(6.0).reshape(2, 3), 7, "x")

    def boom(*a):
        raise RuntimeError("kernel argument rejected")

    with pytest.raises(RuntimeError, match="rejected"):
        diff_tritracer._call_with_snapshot(boom, args, True, "snapshot_fw.dump", "forward")
    saved = torch.load("snapshot_fw.dump")
    assert torch.equal(saved[0], args[0]) and saved[1:] == (7, "x")
    os.remove("snapshot_fw.dump")
    with pytest.raises(RuntimeError):
        diff_tritracer._call_with_snapshot(boom, args, False, "snapshot_fw.dump", "forward")
    assert not os.path.exists("snapshot_fw.dump")
    # a call that succeeds leaves nothing behind
    assert diff_tritracer._call_with_snapshot(lambda *a: a[1] + 1, args, True, "snapshot_fw.dump", "forward") == 8
    assert not os.path.exists("snapshot_fw.dump")


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_tracer_forward_snapshot_on_gpu(tmp_path, monkeypatch):
    from gpu_helpers import T, settings
    from scenes_for_tests import dense_scene, dense_view

    monkeypatch.chdir(tmp_path)
    sc = dense_scene(seed=1, P=200)
    ro, rd = dense_view(H=8, W=8)
    tracer = diff_tritracer.Tracer("forward.ptx", "backward.ptx")
    st = settings(sh_degree=4, debug=True)  # rejected by the tracer
    with pytest.raises(RuntimeError, match="sh_degree"):
        tracer(T(ro), T(rd), T(sc.verts.reshape(-1)), T(sc.sigma), T(sc.num_points), T(sc.cumsum), sc.P,
               T(sc.opacities), torch.zeros(sc.P, device="cuda"), torch.zeros(sc.P, device="cuda"), T(sc.shs), None, st)
    saved = torch.load("snapshot_fw.dump")
    assert isinstance(saved, tuple) and all(not (isinstance(v, torch.Tensor) and v.is_cuda) for v in saved)
    np.testing.assert_array_equal(saved[0].numpy(), ro)
