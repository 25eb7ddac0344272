"""Small seeded scenes shared by the tests (sizes the oracle finishes in
seconds)."""
import numpy as np

from diff_tritracer import scenes


def dense_scene(seed=1, P=3000):
    # a compact cloud of large triangles: many rays see > 16 hits, so the
    # chunked re-trace and the transmittance cut-off are both exercised
    return scenes.make_scene(P, seed=seed, center_std=0.15, edge_range=(0.05, 0.3))


def dense_view(H=48, W=64, origin=(0.3, 0.4, 3.0), fov=12.0):
    cam = scenes.look_at_camera(list(origin), H, W, fov_deg=fov)
    return scenes.camera_rays(cam)


def sphere_extra(samples=3):
    # analytic sphere [r, cx, cy, cz, samples] beside the cloud
    return np.array([0.35, 0.45, 0.0, 0.6, samples], np.float32)
