"""The byte model behind the roofline figures and the autotune cache, on the
host (no GPU).

* Compulsory bytes of a batched time step: 40 B per shot cell plus 20 B per
  model cell under any window (the material is read once and shared), the
  batched form of the per-cell figure; overlapping windows count their shared
  rows once.
* The autotune cache survives processes that store at the same time: every
  reader gets a whole JSON document (each process writes its own temporary
  file and renames it).
"""
import json
import multiprocessing as mp
import os

import numpy as np

from taichirtm_b200 import autotune
from taichirtm_b200.benchmarks import _step_bytes, _union_cells
from taichirtm_b200.plan import ShotGeometry


def _shot(x0, nx):
    z = np.zeros((1, 2), np.int32)
    return ShotGeometry(x0, nx, z, z)


def test_union_counts_overlapping_windows_once():
    shots = [_shot(0, 10), _shot(5, 10), _shot(30, 4)]
    assert _union_cells(shots, 7) == (15 + 4) * 7


def test_step_bytes_batched_form():
    nz = 11
    shots = [_shot(0, 20), _shot(10, 20)]
    cells = 40 * nz
    union = 30 * nz
    assert _step_bytes(shots, nz) == 40 * cells + 20 * union
    # one shot alone: the per-cell figure of 60 B
    assert _step_bytes([_shot(3, 9)], nz) == 60 * 9 * nz


def _store_many(path, tag, n):
    os.environ["TAICHIRTM_B200_CACHE"] = path
    for i in range(n):
        c = autotune._load()
        c[f"{tag}{i}"] = dict(tune=dict(vec=2, rows=i), ms_per_step=float(i))
        autotune._store(c)


def test_autotune_cache_concurrent_stores(tmp_path):
    path = str(tmp_path / "tune.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_store_many, args=(path, t, 25)) for t in ("a", "b")]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    with open(path) as f:
        cache = json.load(f)  # a whole document, whichever process stored last
    assert any(k.startswith(("a", "b")) for k in cache)
    assert not [f for f in os.listdir(tmp_path) if f.endswith(".tmp")]
