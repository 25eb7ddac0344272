"""BVH blobs are checked on the host before anything reaches the device
(tt_bvh_load): a blob whose header is right but whose contents are not -
an index out of range, a Morton order that is not a permutation, parent
links that do not match the tree, a wide child reference that does not
point forward - is refused with "corrupted BVH blob", and the handle stays
usable. The valid round trip is covered by test_gpu_parity.py."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from diff_tritracer import _C  # noqa: E402
from gpu_helpers import T  # noqa: E402
from scenes_for_tests import dense_scene  # noqa: E402

HEADER = 24  # magic[8], P, nw (int32), pad (int64)


def sections(blob):
    """Byte offsets of the blob's sections (the layout bvh.cu writes)."""
    P, nw = np.frombuffer(blob, np.int32, 2, 8)
    b = max(int(P) - 1, 1)
    off, out = HEADER, {}
    for name, n in (("vals", 4 * P), ("topo", 16 * b), ("bparent", 4 * b), ("lparent", 4 * P),
                    ("wsrc", 32 * nw), ("wref", 32 * nw)):
        out[name] = (off, int(n))
        off += int(n)
    assert off == len(blob)
    return int(P), int(nw), out


def patched(blob, name, index, value, dtype=np.int32):
    _, _, sec = sections(blob)
    arr = bytearray(blob)
    view = np.frombuffer(arr, dtype, sec[name][1] // 4, sec[name][0])
    view[index] = value
    return bytes(arr)


@pytest.fixture(scope="module")
def saved():
    sc = dense_scene(seed=2, P=2500)
    tr = _C.OptixTracer()
    tr.build_tri_accel(T(sc.verts), T(sc.cumsum), sc.P, True)
    return sc, tr.save_bvh()


def corruptions(blob):
    P, nw, sec = sections(blob)
    wref = np.frombuffer(blob, np.uint32, sec["wref"][1] // 4, sec["wref"][0])
    inner = int(np.nonzero((wref & 0x80000000) == 0)[0][0])  # a slot that holds a wide child
    leaf = int(np.nonzero(((wref & 0x80000000) != 0) & (wref != 0x7FFFFFFF))[0][0])
    topo = np.frombuffer(blob, np.int32, sec["topo"][1] // 4, sec["topo"][0]).reshape(-1, 4)
    child = int(topo[0, 0]) if topo[0, 0] >= 0 else int(topo[0, 1])
    yield "wide child pointing back", patched(blob, "wref", inner, inner // 8, np.uint32)
    yield "leaf range past P", patched(blob, "wref", leaf, 0x80000000 | (2 << 28) | (P - 1), np.uint32)
    yield "Morton order not a permutation", patched(blob, "vals", 1, int(np.frombuffer(blob, np.uint32, 1, HEADER)[0]))
    yield "parent link off the tree", patched(blob, "bparent", child, 5 if child != 5 else 6)
    yield "slot source out of range", patched(blob, "wsrc", 3, P + 7)


def test_corrupted_blobs_are_refused(saved):
    sc, blob = saved
    tr = _C.OptixTracer()
    n = 0
    for what, bad in corruptions(blob):
        with pytest.raises(RuntimeError, match="corrupted BVH blob"):
            tr.load_bvh(bad, T(sc.verts), T(sc.cumsum), sc.P)
        n += 1
    assert n == 5
    tr.load_bvh(blob, T(sc.verts), T(sc.cumsum), sc.P)  # the intact blob still loads
    tr.device_status()
