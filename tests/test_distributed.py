"""Multi-rank host logic of the shot-sharded path on CPU (gloo, world size 2):
partition, FP64 reduction, and failure agreement (a rank that fails makes
every rank raise instead of hanging in the data collective)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from taichirtm_b200.distributed import run_sharded, shard_shots


def test_shard_shots_partition_is_complete_and_balanced():
    rng = np.random.default_rng(3)
    costs = rng.integers(200, 900, size=64) * 801
    parts = [shard_shots(costs, 4, r) for r in range(4)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.05
    assert shard_shots(costs, 4, 2) == parts[2]  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _shot_image(i):
    g = torch.Generator().manual_seed(1000 + i)
    return torch.randn((3, 12, 9), generator=g, dtype=torch.float64)


def _worker(rank, world, port, fail_rank, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    costs = [5, 9, 2, 7, 7, 3, 8, 1]

    def compute(idx):
        if rank == fail_rank:
            raise FloatingPointError("propagation became non-finite (code 3)")
        acc = torch.zeros((3, 12, 9), dtype=torch.float64)
        for i in idx:
            acc += _shot_image(i)
        return acc

    try:
        total = run_sharded(costs, compute)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), total.numpy())
        result = "ok"
    except Exception as e:  # noqa: BLE001
        result = type(e).__name__
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(result)
    dist.destroy_process_group()


@pytest.mark.parametrize("fail_rank", [-1, 1])
def test_run_sharded_gloo(tmp_path, fail_rank):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), fail_rank, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [open(tmp_path / f"r{r}.txt").read() for r in range(world)]
    if fail_rank < 0:
        assert res == ["ok", "ok"]
        ref = sum(_shot_image(i) for i in range(8)).numpy()
        for r in range(world):
            assert np.allclose(np.load(tmp_path / f"r{r}.npy"), ref, rtol=1e-12, atol=1e-12)
    else:
        # the failing rank re-raises its own error; the other rank learns of it
        # through the status exchange and raises instead of hanging
        assert res[fail_rank] == "FloatingPointError"
        assert res[1 - fail_rank] == "RuntimeError"


def _record_collectives(monkeypatch, backend, fail):
    """run_sharded on a stand-in two-rank group whose all-reduce records
    (device, dtype, shape) and returns the local values."""
    from taichirtm_b200 import distributed as D
    calls = []
    monkeypatch.setattr(D.dist, "get_world_size", lambda group=None: 2)
    monkeypatch.setattr(D.dist, "get_rank", lambda group=None: 0)
    monkeypatch.setattr(D.dist, "get_backend", lambda group=None: backend)
    monkeypatch.setattr(D.dist, "all_reduce",
                        lambda t, op=None, group=None: calls.append((t.device.type, t.dtype, tuple(t.shape))))

    def compute(idx):
        if fail:
            raise FloatingPointError("code 3")
        return torch.ones((3, 4, 5), dtype=torch.float64)
    try:
        D.run_sharded([1, 2, 3], compute)
    except FloatingPointError:
        pass
    return calls


def test_success_and_failure_paths_issue_the_same_status_collective(monkeypatch):
    ok = _record_collectives(monkeypatch, "gloo", fail=False)
    bad = _record_collectives(monkeypatch, "gloo", fail=True)
    assert ok[0] == bad[0] == ("cpu", torch.int64, (1,))  # the status all-reduce, identical on both paths
    assert ok[1] == ("cpu", torch.float64, (3, 4, 5)) and len(bad) == 1  # data only after a clean status


def test_collective_device_follows_the_backend(monkeypatch):
    from taichirtm_b200 import distributed as D
    monkeypatch.setattr(D.dist, "get_backend", lambda group=None: "nccl")
    monkeypatch.setattr(D.torch.cuda, "current_device", lambda: 3)
    assert D.collective_device() == torch.device("cuda", 3)
    monkeypatch.setattr(D.dist, "get_backend", lambda group=None: "gloo")
    assert D.collective_device() == torch.device("cpu")
