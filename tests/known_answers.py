"""Known-answer cases of the trace path: scenes whose images and gradients
follow in closed form from the reference's compositing rules, with no BVH,
intersector or oracle involved.

Geometry. Every triangle is equilateral with inradius r, in a plane z = const,
centred on the z axis; edge A->B lies on x = r, so the incenter's
perpendicular to that edge points along +x. Rays run along -z from
(x, y, z0), so the hit point is (x, y, z) and the hit distance is z0 - z.

Window function (common.h:57-114). The outward edge normals of this triangle
are (1, 0), (-1/2, sqrt 3/2) and (-1/2, -sqrt 3/2), so phi = max_i n_i.p - r
and phi_final = phi / (-r) = 1 - m / r with m = max_i n_i.p. Then
Cx = phi_final ** sigma: 1 at the incenter, 0 on an edge.

SH (common.h:16-55, constants auxiliary.h:13-30). Along d = (0, 0, -1) only
the m = 0 basis functions are non-zero: Y0 = C0, Y2 = -C1 (z = -1),
Y6 = 2 C2[2] (2z^2 - x^2 - y^2 = 2) and Y12 = -2 C3[3] (z(2z^2 - ...) = -2).
Colour = sum_k Y_k sh_k + 0.5, clamped at 0 from below.

Compositing (forward.cu:76-155, closestk.h:17-149). Hits are consumed in
chunks of 16 sorted by t; the next chunk starts at the last hit's t, and with
the closed interval [tmin, tmax] that hit is consumed twice. A hit with
t < 0.2 is skipped (it still fills the chunk); alpha = min(0.99, op * Cx);
alpha < 1/255 is skipped; if T (1 - alpha) < 1e-4 the ray stops without
blending that hit; else w = alpha T, C += w c, N += w n, T *= 1 - alpha.

Adjoint (backward.cu:25-350). For a blended hit, with C, D, N including it:
dL/dalpha = sum_c g_c (T c_c - (Cf_c - C_c)/(1 - alpha))
          + g_D (T t - (Df - D)/(1 - alpha)) + g_N . (T n - (Nf - N)/(1 - alpha)),
where Cf includes T_final bg and Df = 0 (the forward never writes depth).
dL/dop += dL/dalpha Cx; dL/dsigma += op dL/dalpha Cx ln(phi_final);
dL/dsh_k += Y_k w g_c on channels whose colour is not clamped.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from diff_tritracer.scenes import Scene

CHUNK = 16
NEAR = 0.2
ALPHA_MAX = 0.99
ALPHA_MIN = 1.0 / 255.0
T_MIN = 1e-4

C0 = 0.28209479177387814
C1 = 0.4886025119029199
C2_2 = 0.31539156525252005
C3_3 = 0.3731763325901154
# basis values along (0, 0, -1), by coefficient index
Y_AXIS = {0: C0, 2: -C1, 6: 2.0 * C2_2, 12: -2.0 * C3_3}

R_IN = 0.5  # inradius; circumradius 2 r = 1
NORMAL = np.array([0.0, 0.0, 1.0])  # normalize(cross(B - A, C - A))


def triangle(z: float, r: float = R_IN) -> np.ndarray:
    s3 = math.sqrt(3.0)
    return np.array([[r, -s3 * r, z], [r, s3 * r, z], [-2.0 * r, 0.0, z]])


def scene(zs, opacities, sigmas, shs, sh_degree) -> Scene:
    P = len(zs)
    verts = np.concatenate([triangle(float(z)) for z in zs], 0).astype(np.float32)
    return Scene(verts=verts, num_points=np.full(P, 3, np.int32), cumsum=(3 * np.arange(P)).astype(np.int32),
                 opacities=np.asarray(opacities, np.float32).reshape(P, 1),
                 sigma=np.asarray(sigmas, np.float32).reshape(P, 1),
                 shs=np.ascontiguousarray(shs, np.float32), sh_degree=sh_degree)


def rays(points, z0: float):
    """Rays along -z from (x, y, z0), one image row: ([1, n, 3], [1, n, 3])."""
    n = len(points)
    ro = np.zeros((1, n, 3), np.float32)
    ro[0, :, :2] = np.asarray(points, np.float32)
    ro[0, :, 2] = z0
    rd = np.zeros((1, n, 3), np.float32)
    rd[0, :, 2] = -1.0
    return ro, rd


def phi_final(x: float, y: float, r: float = R_IN) -> float:
    s3 = math.sqrt(3.0)
    m = max(x, -0.5 * x + 0.5 * s3 * y, -0.5 * x - 0.5 * s3 * y)
    return 1.0 - m / r


def sh_raw(coeffs: np.ndarray) -> np.ndarray:
    """Unclamped colour along (0, 0, -1) of one triangle's [M, 3] coefficients."""
    out = np.full(3, 0.5)
    for k, y in Y_AXIS.items():
        if k < coeffs.shape[0]:
            out = out + y * coeffs[k].astype(np.float64)
    return out


@dataclass
class Blend:
    prim: int
    t: float
    alpha: float
    T: float  # transmittance before the hit
    cx: float
    phi: float


@dataclass
class RayAnswer:
    color: np.ndarray
    T: float
    normal: np.ndarray
    blends: list = field(default_factory=list)
    terminated: bool = False
    consumed: int = 0  # hits taken from the chunks, duplicates and near-skipped ones included
    depth: float = 0.0  # exact-adjoint forward only: sum w t
    middepth: float = 0.0
    distortion: float = 0.0
    margin: float = math.inf  # smallest relative distance of a decision to its threshold


def chunked(hits, closed: bool):
    """The sequence of hit indices the chunked march consumes (hits sorted by t)."""
    out, start = [], 0
    while True:
        chunk = list(range(start, min(start + CHUNK, len(hits))))
        out.extend(chunk)
        if len(chunk) < CHUNK:
            return out
        start = chunk[-1] if closed else chunk[-1] + 1


def trace_ray(hits, sc: Scene, bg, closed: bool) -> RayAnswer:
    """hits: [(prim, t, x, y)] sorted by t, all on this ray."""
    bg = np.asarray(bg, np.float64)
    C, N, T = np.zeros(3), np.zeros(3), 1.0
    ans = RayAnswer(color=C, T=T, normal=N)
    D, wsum, wt2, mid_set = 0.0, 0.0, 0.0, False
    for idx in chunked(hits, closed):
        ans.consumed += 1
        prim, t, x, y = hits[idx]
        if t < NEAR:
            continue
        ph = phi_final(x, y)
        cx = max(0.0, ph ** float(sc.sigma[prim, 0])) if ph > 0 else 0.0
        alpha = min(ALPHA_MAX, float(sc.opacities[prim, 0]) * cx)
        ans.margin = min(ans.margin, abs(alpha - ALPHA_MIN) / ALPHA_MIN)
        if alpha < ALPHA_MIN:
            continue
        test_T = T * (1.0 - alpha)
        ans.margin = min(ans.margin, abs(test_T - T_MIN) / T_MIN)
        if test_T < T_MIN:
            ans.terminated = True
            break
        w = alpha * T
        ans.blends.append(Blend(prim, t, alpha, T, cx, ph))
        C = C + w * np.maximum(sh_raw(sc.shs[prim]), 0.0)
        N = N + w * NORMAL
        ans.distortion += w * (t * t * wsum - 2.0 * t * D + wt2)
        wsum += w
        D += w * t
        wt2 += w * t * t
        if not mid_set and test_T <= 0.5:
            ans.middepth, mid_set = t, True
        T = test_T
    ans.color, ans.T, ans.normal, ans.depth = C + T * bg, T, N, D
    return ans


def ray_grads(ans: RayAnswer, sc: Scene, bg, g, g_depth, g_normal):
    """Adjoint of one ray (reference semantics, Df = 0): dopac [P], dsigma [P], dsh [P, M, 3]."""
    P, M = sc.P, sc.shs.shape[1]
    dop, dsig, dsh = np.zeros(P), np.zeros(P), np.zeros((P, M, 3))
    g = np.asarray(g, np.float64)
    g_normal = np.asarray(g_normal, np.float64)
    Cf = ans.color
    Nf = ans.normal
    C, N, D = np.zeros(3), np.zeros(3), 0.0
    for b in ans.blends:
        raw = sh_raw(sc.shs[b.prim])
        col = np.maximum(raw, 0.0)
        w = b.alpha * b.T
        C, N, D = C + w * col, N + w * NORMAL, D + w * b.t
        one = 1.0 - b.alpha
        da = float(np.dot(g, b.T * col - (Cf - C) / one))
        da += g_depth * (b.T * b.t - (0.0 - D) / one)
        da += float(np.dot(g_normal, b.T * NORMAL - (Nf - N) / one))
        op = float(sc.opacities[b.prim, 0])
        dop[b.prim] += da * b.cx
        if b.phi > 0:
            dsig[b.prim] += op * da * b.cx * math.log(b.phi)
        for k, y in Y_AXIS.items():
            if k < M:
                dsh[b.prim, k] += y * w * g * (raw >= 0)
    return dop, dsig, dsh


# ---------------------------------------------------------------- the cases
WINDOW_POINTS = [(0.0, 0.0), (0.125, 0.0), (0.25, 0.0), (0.375, 0.0), (-0.25, 0.0), (-0.45, 0.0), (0.1, 0.2),
                 (-0.2, -0.3), (0.5, 0.0), (0.5, 0.6), (0.75, 0.0), (-1.2, 0.0)]


def window_case(sigma=1.5, opacity=0.8, seed=0):
    """One triangle at z = 0, rays at the incenter, inside, on an edge (x = r,
    Cx = 0), beyond a vertex and outside (misses); SH degree 3."""
    rng = np.random.default_rng(seed)
    shs = rng.normal(0.0, 0.1, (1, 16, 3))
    shs[0, 0] = [0.9, 0.4, 0.7]
    sc = scene([0.0], [opacity], [sigma], shs, 3)
    ro, rd = rays(WINDOW_POINTS, 3.0)
    return sc, ro, rd


def window_answers(sc, bg, closed=True):
    out = []
    for x, y in WINDOW_POINTS:
        inside = phi_final(x, y) >= 0.0
        hits = [(0, 3.0, x, y)] if inside else []
        out.append(trace_ray(hits, sc, bg, closed))
    return out


STACK_N = 60
STACK_DZ = 0.05


def stack_case(seed=3):
    """STACK_N identical sheets at z = -0.05 i on the axis (every hit at an
    incenter, Cx = 1 up to rounding). Opacity 0.1 except: sheet 2 below the
    1/255 floor, sheet 5 at 0.05, sheet 7 at 0.6, and sheet 11 clamped to
    0.99 by opacity 1; sheet 4's red channel clamps at 0."""
    rng = np.random.default_rng(seed)
    zs = (-STACK_DZ * np.arange(STACK_N)).astype(np.float32)
    op = np.full(STACK_N, 0.1)
    op[2], op[5], op[7], op[11] = 1.0 / 300.0, 0.05, 0.6, 1.0
    sig = rng.uniform(0.5, 2.0, STACK_N)
    shs = rng.normal(0.0, 0.05, (STACK_N, 16, 3))
    shs[:, 0] = rng.normal(0.6, 0.3, (STACK_N, 3))
    shs[4, 0, 0] = -3.0
    return scene(zs, op, sig, shs, 3), zs


def stack_answer(sc, zs, z0, bg, closed):
    z0 = float(np.float32(z0))
    hits = [(i, z0 - float(z), 0.0, 0.0) for i, z in enumerate(zs) if z0 - float(z) >= 0.0]
    return trace_ray(sorted(hits, key=lambda h: h[1]), sc, bg, closed)


def scaling_of(z0, z):
    """Largest angle, seen from (0, 0, z0), between a vertex and the centroid
    of the sheet at z (circumradius 1)."""
    return math.atan2(2.0 * R_IN, z0 - z)
