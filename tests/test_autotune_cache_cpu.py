"""The autotuner's cache file is written by every rank of a multi-GPU run at
once: concurrent writers never raise and always leave a complete JSON file."""
import json
import multiprocessing as mp
import os

from diff_tritracer.autotune import _store


def _writer(path, rank, n):
    for i in range(n):
        _store(path, {f"rank{rank}": i, "pad": "x" * 4096})


def test_concurrent_cache_writes(tmp_path):
    path = str(tmp_path / "sub" / "autotune.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, r, 200)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    data = json.load(open(path))
    assert data["pad"] == "x" * 4096 and any(k.startswith("rank") for k in data)
    assert not [f for f in os.listdir(tmp_path / "sub") if f.endswith(".tmp")]
