"""The oracle's secondary-ray semantics (CPU): with no dielectric triangles
and a constant environment it is the plain trace; the spawned rays change
the image; its opacity, sigma and SH gradients match FP64 central finite
differences (the spawn geometry depends on vertices only)."""
import numpy as np
import pytest

from diff_tritracer import scenes
from scenes_for_tests import dense_scene, dense_view


def rel_norm(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-30))

H, W = 24, 32


@pytest.fixture(scope="module")
def setup():
    sc = dense_scene(seed=7, P=1200)
    ro, rd = dense_view(H=H, W=W)
    sec = scenes.secondary_inputs(sc.P, seed=7, p_dielectric=0.3, env_shape=(16, 32), box=3)
    return sc, ro, rd, sec


def test_box_filter_wraps_longitude():
    img = np.zeros((6, 8, 1), np.float32)
    img[2, 0, 0] = 9.0
    out = scenes.box_filter_latlong(img, 3)
    assert np.isclose(out.sum(), 9.0) and out[2, 7, 0] == 1.0 and out[2, 1, 0] == 1.0


def test_reduces_to_plain(oracle, setup):
    sc, ro, rd, sec = setup
    bg = np.array([0.2, 0.4, 0.6], np.float32)
    flat = dict(sec, material=np.zeros(sc.P, np.int32), env=np.broadcast_to(bg, (4, 8, 3)).copy())
    a = oracle.forward(sc, ro, rd, bg=bg, precision=64, exact=True, canonical=True, nthreads=8)
    b = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, nthreads=8, secondary=flat)
    np.testing.assert_allclose(b.color, a.color, rtol=0, atol=1e-12)
    np.testing.assert_allclose(b.others, a.others, rtol=0, atol=1e-12)
    np.testing.assert_array_equal(b.density, a.density)


def test_spawned_rays_change_the_image(oracle, setup):
    sc, ro, rd, sec = setup
    none = dict(sec, material=np.zeros(sc.P, np.int32))
    a = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, nthreads=8, secondary=none)
    b = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, nthreads=8, secondary=sec)
    changed = np.abs(a.color - b.color).max(0) > 1e-3
    assert changed.mean() > 0.2
    # side outputs come from the primary ray only: alpha is unchanged
    np.testing.assert_allclose(a.others[1], b.others[1], rtol=0, atol=1e-12)


def test_gradients_match_finite_differences(oracle, setup):
    sc, ro, rd, sec = setup
    g, go = scenes.upstream_grads(H, W, seed=5, others_std=1.0)
    go[0] = 0.0
    kw = dict(precision=64, exact=True, canonical=True, nthreads=8, secondary=sec)
    f = oracle.forward(sc, ro, rd, **kw)
    b = oracle.backward(sc, ro, rd, f.color, f.others, g, go, **kw)

    def loss():
        r = oracle.forward(sc, ro, rd, **kw)
        return float((r.color * g).sum() + (r.others[2:5] * go[2:5]).sum())

    for field, grad in (("opacities", b.dopac), ("sigma", b.dsigma), ("shs", b.dsh)):
        arr = getattr(sc, field).reshape(-1)
        picks = np.argsort(-np.abs(grad.reshape(-1)))[:8]
        errs = []
        for i in picks:
            x0 = arr[i]
            xp, xm = np.float32(x0 + 1e-4), np.float32(x0 - 1e-4)
            arr[i] = xp
            lp = loss()
            arr[i] = xm
            lm = loss()
            arr[i] = x0
            num = (lp - lm) / (float(xp) - float(xm))
            ana = float(grad.reshape(-1)[i])
            errs.append(abs(num - ana) / max(abs(ana), abs(num), 1e-12))
        errs = np.array(errs)
        print(field, np.round(np.sort(errs), 6))
        assert np.median(errs) < 1e-4 and (errs < 1e-4).mean() >= 0.75, (field, errs)


def test_env_and_ior_gradients_match_finite_differences(oracle, setup):
    """The environment map enters each ray's radiance linearly (T env(d)),
    so its gradient must match central differences to rounding. The IOR
    gradient goes through Schlick's Fresnel share with the bent directions
    held constant: it is checked against differences over the oracle's
    Fresnel-only IOR (the test hook `ior_fresnel`)."""
    sc, ro, rd, sec = setup
    g, go = scenes.upstream_grads(H, W, seed=6, others_std=1.0)
    go[0] = 0.0
    kw = dict(precision=64, exact=True, canonical=True, nthreads=8)
    f = oracle.forward(sc, ro, rd, secondary=sec, **kw)
    b = oracle.backward(sc, ro, rd, f.color, f.others, g, go, secondary=sec, **kw)
    assert b.denv.shape == sec["env"].shape and b.dior.shape == (sc.P,)
    assert np.abs(b.denv).max() > 0 and np.abs(b.dior).max() > 0

    def loss(s):
        r = oracle.forward(sc, ro, rd, secondary=s, **kw)
        return float((r.color * g).sum() + (r.others[2:5] * go[2:5]).sum())

    env = sec["env"].astype(np.float32).copy()
    for i in np.argsort(-np.abs(b.denv.reshape(-1)))[:8]:
        e = env.reshape(-1).copy()
        x0 = e[i]
        e[i] = np.float32(x0 + 1e-2)
        lp = loss(dict(sec, env=e.reshape(env.shape)))
        e[i] = np.float32(x0 - 1e-2)
        lm = loss(dict(sec, env=e.reshape(env.shape)))
        num = (lp - lm) / (float(np.float32(x0 + 1e-2)) - float(np.float32(x0 - 1e-2)))
        ana = float(b.denv.reshape(-1)[i])
        assert abs(num - ana) <= 1e-6 * max(abs(ana), 1e-9) + 1e-12, (i, num, ana)

    ior = sec["ior"].astype(np.float32)
    errs = []
    for i in np.argsort(-np.abs(b.dior))[:8]:
        fr = ior.copy()
        fr[i] = np.float32(ior[i] + 1e-4)
        lp = loss(dict(sec, ior_fresnel=fr))
        fr[i] = np.float32(ior[i] - 1e-4)
        lm = loss(dict(sec, ior_fresnel=fr))
        num = (lp - lm) / (float(np.float32(ior[i] + 1e-4)) - float(np.float32(ior[i] - 1e-4)))
        ana = float(b.dior[i])
        errs.append(abs(num - ana) / max(abs(ana), abs(num), 1e-12))
    errs = np.array(errs)
    print("ior", np.round(np.sort(errs), 6))
    assert np.median(errs) < 1e-4 and (errs < 1e-3).all(), errs
    # without the hook the oracle's IOR is both the Fresnel and the bending one
    same = oracle.forward(sc, ro, rd, secondary=dict(sec, ior_fresnel=ior.copy()), **kw)
    np.testing.assert_array_equal(same.color, f.color)


def test_exact_adjoint_matches_finite_differences(oracle):
    """With the exact adjoint the vertex gradient follows the full chain rule
    (incenter distance, hit point, face normal). The spawn geometry still
    depends on the dielectric triangles' vertices and is held constant, so
    the check covers the vertices of triangles that spawn nothing: moving
    one of them moves no spawned ray. Depth is 0 in these passes, so only
    colour and normal carry upstream gradients."""
    sc = scenes.make_scene(1000, seed=9, center_std=0.12, edge_range=(0.04, 0.15))
    cam = scenes.look_at_camera([0.4, 0.3, 3.0], H, W, fov_deg=10.0)
    ro, rd = scenes.camera_rays(cam)
    sec = scenes.secondary_inputs(sc.P, seed=9, p_dielectric=0.3, env_shape=(16, 32), box=3)
    g, go = scenes.upstream_grads(H, W, seed=4, others_std=1.0)
    go[0] = 0.0
    go[5:7] = 0.0
    kw = dict(precision=64, exact=True, canonical=True, nthreads=8, exact_adjoint=True, secondary=sec)
    f = oracle.forward(sc, ro, rd, **kw)
    b = oracle.backward(sc, ro, rd, f.color, f.others, g, go, **kw)
    ref_style = oracle.backward(sc, ro, rd, f.color, f.others, g, go, **dict(kw, exact_adjoint=False))
    assert rel_norm(b.dtri, ref_style.dtri) > 1e-2  # the chain rule's extra terms are not small

    def loss():
        r = oracle.forward(sc, ro, rd, **kw)
        return float((r.color * g).sum() + (r.others[2:5] * go[2:5]).sum())

    plain_vertex = np.zeros(b.dtri.shape[0], bool)
    for p in np.nonzero(sec["material"] == 0)[0]:
        plain_vertex[sc.cumsum[p]:sc.cumsum[p] + sc.num_points[p]] = True
    grad = np.where(plain_vertex[:, None], b.dtri, 0.0)
    arr = sc.verts.reshape(-1)
    errs = []
    for i in np.argsort(-np.abs(grad.reshape(-1)))[:12]:
        x0 = arr[i]
        xp, xm = np.float32(x0 + 1e-5), np.float32(x0 - 1e-5)
        arr[i] = xp
        lp = loss()
        arr[i] = xm
        lm = loss()
        arr[i] = x0
        num = (lp - lm) / (float(xp) - float(xm))
        ana = float(grad.reshape(-1)[i])
        errs.append(abs(num - ana) / max(abs(ana), abs(num), 1e-12))
    errs = np.array(errs)
    print("verts (exact, non-spawning triangles)", np.round(np.sort(errs), 6))
    assert np.median(errs) < 1e-3 and (errs < 1e-2).mean() >= 0.75, errs
