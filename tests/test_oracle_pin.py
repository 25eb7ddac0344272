"""Pins the oracle (a CPU restatement of the reference's trace path) against
the reference's own device code.

* With the reference's sources present, `make -C oracle ref` compiles
  tritracer/{forward,backward,reflect,refract,envlight}.cu for the host with a
  stand-in for the OptiX device API (oracle/refshim); the oracle's FP32
  instantiation must then match it BIT FOR BIT on every output, in both tmin
  conventions.
* Without them, the committed fixtures (tests/golden/make_golden.py) carry the
  same check.
* The FP64 oracle must agree with the FP32 one to FP32 rounding.
"""
import os

import numpy as np
import pytest

from scenes_for_tests import dense_scene, dense_view, sphere_extra
from diff_tritracer import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_host_fp32.npz")


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.fixture(scope="module")
def case():
    sc = dense_scene(seed=1, P=3000)
    ro, rd = dense_view(H=48, W=64)
    return sc, ro, rd


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("incl", [True, False])
def test_forward_bitwise_vs_reference_code(oracle, reference, case, variant, incl):
    sc, ro, rd = case
    bg = np.array([0.2, 0.1, 0.05], np.float32)
    a = oracle.forward(sc, ro, rd, bg=bg, extra=sphere_extra(), variant=variant, tmin_inclusive=incl)
    b = reference.forward(sc, ro, rd, bg=bg, extra=sphere_extra(), variant=variant, tmin_inclusive=incl)
    assert a.color.mean() > 0.05  # the view actually sees the cloud
    for n in ("color", "others", "scaling", "density", "max_blending"):
        assert bits_equal(getattr(a, n), getattr(b, n)), n


@pytest.mark.parametrize("incl", [True, False])
def test_backward_bitwise_vs_reference_code(oracle, reference, case, incl):
    sc, ro, rd = case
    g, go = scenes.upstream_grads(48, 64, seed=2, others_std=1.0)
    f = reference.forward(sc, ro, rd, tmin_inclusive=incl)
    a = oracle.backward(sc, ro, rd, f.color, f.others, g, go, tmin_inclusive=incl)
    b = reference.backward(sc, ro, rd, f.color, f.others, g, go, tmin_inclusive=incl)
    assert np.abs(b.dopac).max() > 0
    for n in ("dtri", "dsigma", "dopac", "dsh"):
        assert bits_equal(getattr(a, n), getattr(b, n)), n


def test_forward_exercises_chunking_and_cutoff(oracle, case):
    sc, ro, rd = case
    r = oracle.forward(sc, ro, rd, record=96)
    assert (r.rec_count > 16).mean() > 0.2  # re-traced chunks
    assert (r.others[1] > 1 - 1.1e-4).any()  # transmittance cut-off reached
    a = oracle.forward(sc, ro, rd, tmin_inclusive=True)
    b = oracle.forward(sc, ro, rd, tmin_inclusive=False)
    # the closed lower bound re-visits the last hit of every full chunk
    assert np.abs(a.color - b.color).max() > 1e-3


def test_golden_fixtures(oracle):
    gold = np.load(GOLDEN)
    sc = dense_scene(seed=1, P=800)
    ro, rd = dense_view(H=24, W=32)
    g, go = scenes.upstream_grads(24, 32, seed=3, others_std=1.0)
    bg = np.array([0.1, 0.2, 0.3], np.float32)
    for name, variant, incl in [("plain_incl", 0, True), ("plain_excl", 0, False), ("reflect", 1, True),
                                ("refract", 2, True), ("envlight", 3, True)]:
        f = oracle.forward(sc, ro, rd, bg=bg, extra=sphere_extra(), variant=variant, tmin_inclusive=incl)
        assert bits_equal(f.color, gold[f"{name}/color"]), name
        if variant == 0:
            for n in ("others", "scaling", "density", "max_blending"):
                assert bits_equal(getattr(f, n), gold[f"{name}/{n}"]), (name, n)
            b = oracle.backward(sc, ro, rd, f.color, f.others, g, go, bg=bg, tmin_inclusive=incl)
            for n in ("dtri", "dsigma", "dopac", "dsh"):
                assert bits_equal(getattr(b, n), gold[f"{name}/{n}"]), (name, n)


def test_fp64_agrees_with_fp32(oracle, case):
    sc, ro, rd = case
    a = oracle.forward(sc, ro, rd, canonical=True)
    r = oracle.forward(sc, ro, rd, precision=64, exact=True, canonical=True, record=4)
    ok = r.margin > 1e-3  # rays with no decision near a threshold
    err = np.abs(a.color - r.color)[:, ok.reshape(a.color.shape[1:])]
    assert ok.mean() > 0.9
    assert err.max() < 2e-3  # FP32 hit points: ~1e-4 relative on small triangles
    assert np.sqrt((err ** 2).mean()) < 2e-5


def test_multithreaded_matches_single(oracle, case):
    sc, ro, rd = case
    a = oracle.forward(sc, ro, rd, nthreads=1)
    b = oracle.forward(sc, ro, rd, nthreads=4)
    assert bits_equal(a.color, b.color) and bits_equal(a.max_blending, b.max_blending)


@pytest.mark.parametrize("incl", [True, False], ids=["closed", "open"])
def test_reference_queries_equal_the_hit_stream(oracle, reference, case, incl):
    """The k-closest queries the reference's own any-hit program answers
    (tritracer/closestk.h:17-149, logged per ray) hold, query by query, the
    same hits as the (t, id)-ordered hit stream of the restated intersector
    and BVH, except for the order inside groups of equal t. The GPU test
    tests/test_gpu_vs_reference.py makes the same check against the GPU's
    hit stream."""
    from ref_chunks import compare_chunks

    sc, ro, rd = case
    f = reference.forward(sc, ro, rd, tmin_inclusive=incl, chunks=8)
    ids, ts, cnt = oracle.hit_stream(sc, ro, rd, max_hits=256, nthreads=8)
    assert (f.chunk_count > 1).mean() > 0.2  # re-traced chunks are logged too
    n, _ = compare_chunks(f.chunk_ids, f.chunk_tmin, f.chunk_count, ids, ts, cnt, incl, 256)
    assert n > 3000
