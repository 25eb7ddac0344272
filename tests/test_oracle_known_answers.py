"""The oracle against closed-form answers (tests/known_answers.py): the window
function on an equilateral triangle (Cx = 1 at the incenter, 0 on an edge,
phi_final ** sigma between), SH along an axis with its clamp at 0, and a
stack of 60 sheets on one ray that exercises the chunked march (the closed
interval consumes the last hit of every full chunk twice), the near cut-off,
the 1/255 floor, the 0.99 clamp and the 1e-4 termination, with the
adjoint's reference semantics (the depth term with D_final = 0)."""
import numpy as np
import pytest

import known_answers as ka

BG = np.array([0.1, 0.2, 0.3])
RTOL, ATOL = 1e-5, 1e-6


def close(a, b, rtol=RTOL, atol=ATOL):
    np.testing.assert_allclose(np.asarray(a, np.float64), np.asarray(b, np.float64), rtol=rtol, atol=atol)


def upstream(n, seed):
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(3, 1, n)).astype(np.float32)
    go = np.zeros((7, 1, n), np.float32)
    go[0] = rng.normal(size=(1, n))
    go[2:5] = rng.normal(size=(3, 1, n))
    return g, go


def expected_grads(answers, sc, g, go):
    P, M = sc.P, sc.shs.shape[1]
    dop, dsig, dsh = np.zeros(P), np.zeros(P), np.zeros((P, M, 3))
    for i, a in enumerate(answers):
        o, s, h = ka.ray_grads(a, sc, BG, g[:, 0, i], float(go[0, 0, i]), go[2:5, 0, i])
        dop, dsig, dsh = dop + o, dsig + s, dsh + h
    return dop, dsig, dsh


def test_model_cases_are_well_posed():
    sc, ro, rd = ka.window_case()
    ans = ka.window_answers(sc, BG)
    alphas = [a.blends[0].alpha if a.blends else 0.0 for a in ans]
    assert alphas[0] == pytest.approx(0.8)  # incenter: Cx = 1
    assert sum(a > ka.ALPHA_MIN for a in alphas) >= 6 and sum(not a.blends for a in ans) >= 4
    assert min(a.margin for a in ans) > 1e-3
    sc, zs = ka.stack_case()
    for z0 in (3.0, -0.225):
        for closed in (True, False):
            a = ka.stack_answer(sc, zs, z0, BG, closed)
            prims = [b.prim for b in a.blends]
            assert a.terminated and len(prims) > 2 * ka.CHUNK and a.margin > 1e-3
            assert (len(prims) != len(set(prims))) == closed  # duplicates only in the closed interval
            assert 2 not in prims and 11 in prims  # the floor and the clamp
    near = ka.stack_answer(sc, zs, -0.225, BG, True)
    assert near.blends[0].prim == 9  # sheets 5..8 lie within 0.2 of the origin


@pytest.mark.parametrize("precision,exact", [(32, False), (64, False), (64, True)])
def test_window_function_and_sh(oracle, precision, exact):
    sc, ro, rd = ka.window_case()
    ans = ka.window_answers(sc, BG)
    f = oracle.forward(sc, ro, rd, bg=BG, precision=precision, exact=exact)
    for i, a in enumerate(ans):
        close(f.color[:, 0, i], a.color)
        close(f.others[1, 0, i], 1.0 - a.T)
        close(f.others[2:5, 0, i], a.normal)
        assert np.all(f.others[[0, 5, 6], 0, i] == 0)  # depth, middepth, distortion are never written
        if not a.blends:
            close(f.color[:, 0, i], BG.astype(np.float32), rtol=0, atol=0)
    close(f.max_blending[0], max(a.blends[0].alpha for a in ans if a.blends))
    assert f.density[0] == 1


@pytest.mark.parametrize("precision", [32, 64])
def test_window_adjoint(oracle, precision):
    sc, ro, rd = ka.window_case()
    ans = ka.window_answers(sc, BG)
    g, go = upstream(ro.shape[1], seed=4)
    f = oracle.forward(sc, ro, rd, bg=BG, precision=precision)
    b = oracle.backward(sc, ro, rd, f.color, f.others, g, go, bg=BG, precision=precision)
    dop, dsig, dsh = expected_grads(ans, sc, g, go)
    assert abs(dsig[0]) > 0.1
    close(b.dopac, dop)
    close(b.dsigma, dsig)
    close(b.dsh, dsh, atol=1e-6)


@pytest.mark.parametrize("closed", [True, False], ids=["closed", "open"])
@pytest.mark.parametrize("z0", [3.0, -0.225], ids=["above", "inside"])
def test_stack_of_sheets(oracle, z0, closed):
    sc, zs = ka.stack_case()
    a = ka.stack_answer(sc, zs, z0, BG, closed)
    ro, rd = ka.rays([(0.0, 0.0)], z0)
    f = oracle.forward(sc, ro, rd, bg=BG, tmin_inclusive=closed)
    close(f.color[:, 0, 0], a.color)
    close(f.others[1, 0, 0], 1.0 - a.T)
    close(f.others[2:5, 0, 0], a.normal)
    blended = sorted({b.prim for b in a.blends})
    want_maxb = np.zeros(sc.P)
    for b in a.blends:
        want_maxb[b.prim] = max(want_maxb[b.prim], b.alpha * b.T)
    close(f.max_blending, want_maxb)
    want_density = np.zeros(sc.P)
    want_density[blended] = 1
    np.testing.assert_array_equal(f.density, want_density)
    want_scaling = np.zeros(sc.P)
    for p in blended:
        want_scaling[p] = ka.scaling_of(z0, float(zs[p]))
    close(f.scaling, want_scaling)

    g, go = upstream(1, seed=5)
    bw = oracle.backward(sc, ro, rd, f.color, f.others, g, go, bg=BG, tmin_inclusive=closed)
    dop, dsig, dsh = expected_grads([a], sc, g, go)
    close(bw.dopac, dop, atol=1e-5)
    close(bw.dsigma, dsig, atol=1e-5)  # phi_final = 1 at the incenters: ln 1 = 0 up to rounding
    close(bw.dsh, dsh, atol=1e-6)


def test_stack_exact_forward_outputs(oracle):
    """exact_adjoint's forward writes depth = sum w t, middepth (t of the hit
    after which T <= 0.5) and distortion sum_{i<j} w_i w_j (t_i - t_j)^2."""
    sc, zs = ka.stack_case()
    a = ka.stack_answer(sc, zs, 3.0, BG, True)
    ro, rd = ka.rays([(0.0, 0.0)], 3.0)
    f = oracle.forward(sc, ro, rd, bg=BG, precision=64, exact=True, exact_adjoint=True)
    ts = np.array([b.t for b in a.blends])
    ws = np.array([b.alpha * b.T for b in a.blends])
    brute = sum(ws[i] * ws[j] * (ts[i] - ts[j]) ** 2 for i in range(len(ts)) for j in range(i))
    close(a.distortion, brute, rtol=1e-12)
    close(f.others[0, 0, 0], a.depth)
    close(f.others[5, 0, 0], a.middepth)
    close(f.others[6, 0, 0], a.distortion)
    close(f.color[:, 0, 0], a.color)


@pytest.mark.parametrize("closed", [True, False], ids=["closed", "open"])
def test_reference_code_gives_the_known_answers(reference, closed):
    """The reference's own device code, built for the host, on the same cases."""
    sc, ro, rd = ka.window_case()
    ans = ka.window_answers(sc, BG, closed)
    g, go = upstream(ro.shape[1], seed=4)
    f = reference.forward(sc, ro, rd, bg=BG, tmin_inclusive=closed)
    for i, a in enumerate(ans):
        close(f.color[:, 0, i], a.color)
        close(f.others[1:5, 0, i], np.concatenate([[1.0 - a.T], a.normal]))
    b = reference.backward(sc, ro, rd, f.color, f.others, g, go, bg=BG, tmin_inclusive=closed)
    for got, want in zip((b.dopac, b.dsigma, b.dsh), expected_grads(ans, sc, g, go)):
        close(got, want)
    sc, zs = ka.stack_case()
    for z0 in (3.0, -0.225):
        a = ka.stack_answer(sc, zs, z0, BG, closed)
        ro, rd = ka.rays([(0.0, 0.0)], z0)
        f = reference.forward(sc, ro, rd, bg=BG, tmin_inclusive=closed)
        close(f.color[:, 0, 0], a.color)
        close(f.others[1, 0, 0], 1.0 - a.T)
        g, go = upstream(1, seed=5)
        b = reference.backward(sc, ro, rd, f.color, f.others, g, go, bg=BG, tmin_inclusive=closed)
        for got, want in zip((b.dopac, b.dsigma, b.dsh), expected_grads([a], sc, g, go)):
            close(got, want, atol=1e-5)
