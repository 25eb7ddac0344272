"""Regenerates the golden fixtures in this directory from the host build of
the reference's own device sources (oracle/_ref, built by `make -C oracle
ref` from the reference's files). The fixtures let the oracle be checked
against the reference's arithmetic where the reference's sources are absent.

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "diff-triangle-tracer_b200"), os.path.join(ROOT, "tests")]

from oracle.pyoracle import Reference  # noqa: E402
from scenes_for_tests import dense_scene, dense_view, sphere_extra  # noqa: E402
from diff_tritracer import scenes  # noqa: E402

CASES = [
    # name, variant, tmin_inclusive
    ("plain_incl", 0, True),
    ("plain_excl", 0, False),
    ("reflect", 1, True),
    ("refract", 2, True),
    ("envlight", 3, True),
]


def main():
    ref = Reference()
    sc = dense_scene(seed=1, P=800)
    ro, rd = dense_view(H=24, W=32)
    g, go = scenes.upstream_grads(24, 32, seed=3, others_std=1.0)
    bg = np.array([0.1, 0.2, 0.3], np.float32)
    out = {}
    for name, variant, incl in CASES:
        f = ref.forward(sc, ro, rd, bg=bg, extra=sphere_extra(), variant=variant, tmin_inclusive=incl)
        out[f"{name}/color"] = f.color
        if variant == 0:
            out[f"{name}/others"] = f.others
            out[f"{name}/scaling"] = f.scaling
            out[f"{name}/density"] = f.density
            out[f"{name}/max_blending"] = f.max_blending
            b = ref.backward(sc, ro, rd, f.color, f.others, g, go, bg=bg, tmin_inclusive=incl)
            out[f"{name}/dtri"] = b.dtri
            out[f"{name}/dsigma"] = b.dsigma
            out[f"{name}/dopac"] = b.dopac
            out[f"{name}/dsh"] = b.dsh
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_host_fp32.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
