"""Seeded synthetic scenes and pinhole cameras for tests and benchmarks.

The reference ships no data set and no scene generator; these inputs follow
the benchmark configurations' description of the workload:

* centres ~ N(0, 0.5^2 I3); a uniformly random rotation per triangle;
* an equilateral-ish template whose three corner radii come from edge lengths
  drawn log-uniformly in [0.005, 0.05];
* opacity = sigmoid(N(0, 1)); SH degree 3, DC ~ N(0.5, 0.2^2), higher bands
  ~ N(0, 0.05^2); sigma ~ U[0.5, 2];
* pinhole cameras on a sphere of radius 3 looking at the origin, fov 50 deg.

Everything is float32 / int32 numpy, in the per-triangle layout the tracer
takes (tritracer/params.h:15-62 in the reference): vertices [3P, 3] with
triangle i at rows cumsum[i]..cumsum[i]+2, SH [P, 16, 3] coefficient-major.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Scene:
    verts: np.ndarray  # [3P, 3] float32
    num_points: np.ndarray  # [P] int32 (always 3)
    cumsum: np.ndarray  # [P] int32 exclusive prefix sum of num_points
    opacities: np.ndarray  # [P, 1] float32, already activated
    sigma: np.ndarray  # [P, 1] float32
    shs: np.ndarray  # [P, M, 3] float32
    sh_degree: int

    @property
    def P(self) -> int:
        return int(self.cumsum.shape[0])


@dataclass
class Camera:
    origin: np.ndarray  # [3]
    forward: np.ndarray
    right: np.ndarray
    up: np.ndarray
    H: int
    W: int
    fov_deg: float


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def make_scene(P: int, seed: int = 0, sh_degree: int = 3, center_std: float = 0.5,
               edge_range=(0.005, 0.05)) -> Scene:
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, center_std, size=(P, 3))
    R = _random_rotations(rng, P)
    lo, hi = np.log(edge_range[0]), np.log(edge_range[1])
    edges = np.exp(rng.uniform(lo, hi, size=(P, 3)))
    ang = np.deg2rad(np.array([90.0, 210.0, 330.0]))
    radii = edges / np.sqrt(3.0)
    tmpl = np.stack([radii * np.cos(ang), radii * np.sin(ang), np.zeros_like(radii)], axis=-1)  # [P,3,3]
    verts = centers[:, None, :] + np.einsum("pij,pkj->pki", R, tmpl)
    opac = 1.0 / (1.0 + np.exp(-rng.normal(size=(P, 1))))
    M = (sh_degree + 1) ** 2
    shs = rng.normal(0.0, 0.05, size=(P, M, 3))
    shs[:, 0, :] = rng.normal(0.5, 0.2, size=(P, 3))
    sigma = rng.uniform(0.5, 2.0, size=(P, 1))
    return Scene(
        verts=verts.reshape(-1, 3).astype(np.float32),
        num_points=np.full(P, 3, dtype=np.int32),
        cumsum=(3 * np.arange(P)).astype(np.int32),
        opacities=opac.astype(np.float32),
        sigma=sigma.astype(np.float32),
        shs=shs.astype(np.float32),
        sh_degree=sh_degree,
    )


def look_at_camera(origin, H: int, W: int, fov_deg: float = 50.0, target=(0.0, 0.0, 0.0)) -> Camera:
    origin = np.asarray(origin, dtype=np.float64)
    fwd = np.asarray(target, dtype=np.float64) - origin
    fwd /= np.linalg.norm(fwd)
    up0 = np.array([0.0, 1.0, 0.0]) if abs(fwd[1]) < 0.99 else np.array([1.0, 0.0, 0.0])
    right = np.cross(fwd, up0)
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    return Camera(origin, fwd, right, up, H, W, fov_deg)


def sphere_cameras(n: int, H: int, W: int, radius: float = 3.0, fov_deg: float = 50.0, seed: int = 0):
    rng = np.random.default_rng(seed + 7919)
    out = []
    for _ in range(n):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        out.append(look_at_camera(radius * v, H, W, fov_deg))
    return out


def camera_rays(cam: Camera):
    """Per-pixel ray origins and unit directions, [H, W, 3] float32 each."""
    H, W = cam.H, cam.W
    tan = np.tan(np.deg2rad(cam.fov_deg) / 2.0)
    aspect = W / H
    xs = (2.0 * (np.arange(W) + 0.5) / W - 1.0) * tan * aspect
    ys = (1.0 - 2.0 * (np.arange(H) + 0.5) / H) * tan
    d = cam.forward[None, None, :] + xs[None, :, None] * cam.right[None, None, :] + ys[:, None, None] * cam.up[None, None, :]
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    o = np.broadcast_to(cam.origin, d.shape)
    return np.ascontiguousarray(o, dtype=np.float32), np.ascontiguousarray(d, dtype=np.float32)


def upstream_grads(H: int, W: int, seed: int = 0, others_std: float = 0.0):
    rng = np.random.default_rng(seed + 104729)
    g = rng.normal(size=(3, H, W)).astype(np.float32)
    go = np.zeros((7, H, W), dtype=np.float32)
    if others_std > 0:
        go[0] = rng.normal(0, others_std, size=(H, W))
        go[2:5] = rng.normal(0, others_std, size=(3, H, W))
    return g, go


def box_filter_latlong(img: np.ndarray, k: int) -> np.ndarray:
    """k x k box filter of a lat-long map [h, w, c]: wraps in longitude,
    clamps (edge-replicates) in latitude."""
    r = k // 2
    pad = np.pad(img, ((r, r), (0, 0), (0, 0)), mode="edge")
    pad = np.concatenate([pad[:, -r:], pad, pad[:, :r]], axis=1).astype(np.float64)
    c = np.cumsum(np.cumsum(pad, 0), 1)
    c = np.pad(c, ((1, 0), (1, 0), (0, 0)))
    h, w = img.shape[:2]
    out = c[k:k + h, k:k + w] - c[:h, k:k + w] - c[k:k + h, :w] + c[:h, :w]
    return (out / (k * k)).astype(np.float32)


def secondary_inputs(P: int, seed: int = 0, p_dielectric: float = 0.2, ior_range=(1.3, 1.6),
                     env_shape=(512, 1024), box: int = 9, max_depth: int = 2) -> dict:
    """Per-triangle dielectric mask (Bernoulli), IOR (uniform) and a lat-long
    environment map (uniform noise, box-filtered) for the secondary-ray
    passes."""
    rng = np.random.default_rng(seed + 31337)
    material = (rng.random(P) < p_dielectric).astype(np.int32)
    ior = rng.uniform(ior_range[0], ior_range[1], P).astype(np.float32)
    env = box_filter_latlong(rng.random((env_shape[0], env_shape[1], 3), dtype=np.float32), box)
    return {"material": material, "ior": ior, "env": env, "max_depth": max_depth}
