"""Edge cases of the CUDA path (through the C ABI):

* an empty scene (P = 0): the image is the background, gradients are empty,
  the handle keeps working;
* degenerate triangles (two or three equal vertices, whose watertight
  determinant is exactly 0 in floating point) are never hit, so a scene with
  them mixed in renders the same image bit for bit and the same gradients
  for the other triangles;
* the far bound t <= 1000 (config.h): of two sheets at t = 999.5 and
  t = 1000.5 only the first is composited;
* images of one pixel, one row and one column match the FP64 oracle.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import known_answers as ka  # noqa: E402
from diff_tritracer import _C, scenes  # noqa: E402
from diff_tritracer.scenes import Scene  # noqa: E402
from gpu_helpers import MARGIN, gpu_backward, gpu_forward, rel_norm, settings  # noqa: E402
from scenes_for_tests import dense_scene, dense_view  # noqa: E402

BG = np.array([0.25, 0.5, 0.75], np.float32)


def test_empty_scene_renders_background():
    sc = Scene(verts=np.zeros((0, 3), np.float32), num_points=np.zeros(0, np.int32), cumsum=np.zeros(0, np.int32),
               opacities=np.zeros((0, 1), np.float32), sigma=np.zeros((0, 1), np.float32),
               shs=np.zeros((0, 16, 3), np.float32), sh_degree=3)
    ro, rd = dense_view(H=12, W=20)
    tr = _C.OptixTracer()
    out = gpu_forward(tr, sc, ro, rd, settings(bg=BG))
    np.testing.assert_array_equal(out["color"], np.broadcast_to(BG[:, None, None], (3, 12, 20)))
    assert np.all(out["others"] == 0) and out["max_blending"].size == 0
    g, go = scenes.upstream_grads(12, 20, seed=1, others_std=1.0)
    grads = gpu_backward(tr, sc, ro, rd, settings(bg=BG), out["color"], out["others"], g, go)
    tr.device_status()
    assert all(x.size == 0 for x in grads.values())
    # the same handle then traces a real scene
    full = dense_scene(seed=1, P=500)
    out = gpu_forward(tr, full, ro, rd, settings(bg=BG))
    tr.device_status()
    assert out["others"][1].max() > 0.5


def with_degenerates(sc, n, seed):
    """`sc` plus n degenerate triangles placed among the others: (a, a, b)
    (half) and (a, a, a) (half), a and b vertices of the scene's triangles."""
    rng = np.random.default_rng(seed)
    P = sc.P
    base = sc.verts.reshape(P, 3, 3)[rng.integers(0, P, n)]
    a, b = base[:, 0], base[:, 1]
    deg = np.stack([a, a, b], 1)
    deg[n // 2:] = a[n // 2:, None, :]
    verts = np.concatenate([sc.verts.reshape(P, 3, 3), deg.astype(np.float32)], 0).reshape(-1, 3)
    M = sc.shs.shape[1]
    return Scene(verts=np.ascontiguousarray(verts), num_points=np.full(P + n, 3, np.int32),
                 cumsum=(3 * np.arange(P + n)).astype(np.int32),
                 opacities=np.concatenate([sc.opacities, np.full((n, 1), 0.9, np.float32)]),
                 sigma=np.concatenate([sc.sigma, np.ones((n, 1), np.float32)]),
                 shs=np.concatenate([sc.shs, np.full((n, M, 3), 0.3, np.float32)]), sh_degree=sc.sh_degree)


@pytest.mark.parametrize("traversal", ["packets", "lanes"])
def test_degenerate_triangles_are_never_hit(traversal):
    sc = dense_scene(seed=4, P=2000)
    dg = with_degenerates(sc, 400, seed=5)
    ro, rd = dense_view(H=40, W=56)
    g, go = scenes.upstream_grads(40, 56, seed=6, others_std=1.0)
    res = []
    for s in (sc, dg):
        tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal)
        f = gpu_forward(tr, s, ro, rd, settings(bg=BG))
        b = gpu_backward(tr, s, ro, rd, settings(bg=BG), f["color"], f["others"], g, go)
        tr.device_status()
        res.append((f, b))
    (f0, b0), (f1, b1) = res
    np.testing.assert_array_equal(f0["color"], f1["color"])
    np.testing.assert_array_equal(f0["others"], f1["others"])
    assert np.all(f1["max_blending"][sc.P:] == 0) and np.all(f1["density"][sc.P:] == 0)
    P = sc.P
    assert np.all(b1["dopac"][P:] == 0) and np.all(b1["dsh"][P:] == 0) and np.all(b1["dtri"][3 * P:] == 0)
    for k, n in (("dopac", P), ("dsigma", P), ("dsh", P), ("dtri", 3 * P)):
        assert rel_norm(b1[k][:n], b0[k]) < 1e-5, k


@pytest.mark.parametrize("traversal", ["packets", "lanes"])
def test_far_bound(oracle, traversal):
    sc = ka.scene([0.5, -0.5], [0.5, 0.5], [1.0, 1.0], np.zeros((2, 16, 3)), 3)  # t = 999.5 and 1000.5
    ro, rd = ka.rays([(0.0, 0.0), (0.1, -0.05)], 1000.0)
    tr = _C.OptixTracer("", "forward.ptx", "backward.ptx", traversal=traversal)
    out = gpu_forward(tr, sc, ro, rd, settings(bg=BG))
    tr.device_status()
    assert out["max_blending"][1] == 0 and out["max_blending"][0] > 0.4
    ref = oracle.forward(sc, ro, rd, bg=BG, precision=64, exact=True, canonical=True)
    np.testing.assert_allclose(out["color"], ref.color, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("shape", [(1, 1), (1, 37), (29, 1)], ids=["pixel", "row", "column"])
def test_thin_images_match_oracle(oracle, shape):
    H, W = shape
    sc = dense_scene(seed=2, P=2000)
    cam = scenes.look_at_camera([0.3, 0.4, 3.0], H, W, fov_deg=6.0)
    ro, rd = scenes.camera_rays(cam)
    tr = _C.OptixTracer()
    out = gpu_forward(tr, sc, ro, rd, settings(bg=BG))
    tr.device_status()
    ref = oracle.forward(sc, ro, rd, bg=BG, precision=64, exact=True, canonical=True, record=64)
    ok = (ref.margin > MARGIN).reshape(H, W)
    assert ok.all()
    np.testing.assert_allclose(out["color"], ref.color, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(out["others"], ref.others, rtol=1e-5, atol=1e-6)
