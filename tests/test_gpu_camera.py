"""Primary rays generated on the device (tt_camera_rays): bit for bit the rays
of the host generator diff_tritracer.scenes.camera_rays, for cameras of
uneven size and field of view in one launch; ViewBatch.set_cameras gives the
same images as uploading those rays; invalid calls raise."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C, scenes  # noqa: E402
from diff_tritracer.batch import ViewBatch  # noqa: E402
from gpu_helpers import DEV, T  # noqa: E402
from scenes_for_tests import dense_scene  # noqa: E402


def cameras():
    cams = scenes.sphere_cameras(3, 37, 53, seed=4)
    cams.append(scenes.look_at_camera([0.3, 0.4, 3.0], 64, 48, fov_deg=12.0))
    cams.append(scenes.look_at_camera([0.0, 3.0, 0.0], 17, 29, fov_deg=80.0))  # looking down: the other up vector
    cams.append(scenes.look_at_camera([-2.0, 0.5, 2.0], 1, 1, fov_deg=30.0))
    return cams


def test_device_rays_equal_host_rays_bit_for_bit():
    tr = _C.OptixTracer()
    cams = cameras()
    got = tr.camera_rays(cams)
    torch.cuda.synchronize()
    for cam, (ro, rd) in zip(cams, got):
        ho, hd = scenes.camera_rays(cam)
        np.testing.assert_array_equal(ro.cpu().numpy().view(np.uint32), ho.view(np.uint32))
        np.testing.assert_array_equal(rd.cpu().numpy().view(np.uint32), hd.view(np.uint32))


def test_batch_set_cameras_matches_uploaded_rays():
    sc = dense_scene(seed=6, P=3000)
    cams = cameras()[3:5]
    shapes = [(c.H, c.W) for c in cams]
    outs = []
    for on_device in (True, False):
        s = dict(triangles_points=T(sc.verts.reshape(-1)), sigma=T(sc.sigma), num_points_per_triangle=T(sc.num_points),
                 cumsum_of_points_per_triangle=T(sc.cumsum), number_of_points=sc.P, shs=T(sc.shs),
                 opacities=T(sc.opacities), scaling=torch.zeros(sc.P, device=DEV),
                 density_factor=torch.zeros(sc.P, device=DEV))
        tr = _C.OptixTracer()
        vb = ViewBatch(tr, shapes, s, 3, torch.zeros(3, device=DEV), graph=True)
        if on_device:
            vb.set_cameras(cams)
        else:
            vb.set_rays([tuple(T(a) for a in scenes.camera_rays(c)) for c in cams])
        vb.step()
        torch.cuda.synchronize()
        tr.device_status()
        outs.append([t.cpu().numpy() for pair in vb.outputs for t in pair])
    assert outs[0][0].max() > 0
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_invalid_camera_calls_raise():
    tr = _C.OptixTracer()
    cam = cameras()[0]
    with pytest.raises(RuntimeError, match="1 to 32 cameras"):
        tr.camera_rays([])
    with pytest.raises(RuntimeError, match="1 to 32 cameras"):
        tr.camera_rays([cam] * 33)
    bad = (torch.empty((cam.H, cam.W + 1, 3), device=DEV), torch.empty((cam.H, cam.W, 3), device=DEV))
    with pytest.raises(RuntimeError, match=r"\[H, W, 3\]"):
        tr.camera_rays([cam], outputs=[bad])
