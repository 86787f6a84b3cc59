"""Launch-shape autotuner for the fused step kernels.

The shape is (vec columns per lane, rows per warp task, warps per CTA, load
pipeline, time steps per launch).  Results never depend on it (every cell's arithmetic is the same; FMA
contraction is off), so the tuner only times: it builds a short plan for each
candidate, times a few forward steps with CUDA events, and caches the best
per (GPU, nz, total window rows, shots, modes) in a JSON file
($TAICHIRTM_B200_CACHE or ~/.cache/taichirtm_b200/autotune.json)."""
import json
import os

import torch

CANDIDATES = [
    # two time steps per launch (temporal blocking; vec 2 or 4); prefetch 3 =
    # material rows through a shared-memory ring (fewer registers, more warps)
    dict(vec=2, rows=24, warps=1, tsteps=2, prefetch=3), dict(vec=2, rows=16, warps=2, tsteps=2, prefetch=3),
    # prefetch 4 = the ring kernel with the task from the block index (one warp per CTA)
    dict(vec=2, rows=24, warps=1, tsteps=2, prefetch=4), dict(vec=2, rows=16, warps=1, tsteps=2, prefetch=4),
    dict(vec=2, rows=32, warps=1, tsteps=2, prefetch=4),
    dict(vec=4, rows=16, warps=1, tsteps=2, prefetch=4), dict(vec=4, rows=24, warps=1, tsteps=2, prefetch=4),
    dict(vec=4, rows=12, warps=1, tsteps=2, prefetch=4),
    dict(vec=2, rows=32, warps=1, tsteps=2, prefetch=3), dict(vec=2, rows=8, warps=2, tsteps=2, prefetch=3),
    dict(vec=2, rows=32, warps=1, tsteps=2), dict(vec=2, rows=16, warps=2, tsteps=2),
    dict(vec=2, rows=8, warps=2, tsteps=2), dict(vec=4, rows=32, warps=1, tsteps=2),
    dict(vec=2, rows=4, warps=4, tsteps=2),
    # one time step per launch
    dict(vec=4, rows=16, warps=1, prefetch=3), dict(vec=4, rows=16, warps=2, prefetch=3),
    dict(vec=4, rows=16, warps=2, prefetch=1),
    dict(vec=4, rows=32, warps=4, prefetch=1), dict(vec=4, rows=16, warps=4, prefetch=1),
    dict(vec=2, rows=16, warps=4, prefetch=1), dict(vec=2, rows=32, warps=4, prefetch=1),
    dict(vec=2, rows=8, warps=4, prefetch=1), dict(vec=1, rows=8, warps=4, prefetch=1),
    dict(vec=1, rows=4, warps=2, prefetch=1), dict(vec=2, rows=4, warps=4, prefetch=1),
    dict(vec=2, rows=16, warps=4, prefetch=0), dict(vec=4, rows=64, warps=4, prefetch=1),
    # small grids (one shot of a few hundred thousand cells): a warp's row loop
    # is a serial chain of dependent loads, so shorter tasks and more warps
    dict(vec=2, rows=2, warps=4, tsteps=2), dict(vec=2, rows=1, warps=4, tsteps=2),
    dict(vec=2, rows=1, warps=1, tsteps=2), dict(vec=2, rows=1, warps=2, tsteps=2),
    dict(vec=2, rows=2, warps=2, tsteps=2),
    dict(vec=1, rows=2, warps=4, prefetch=1), dict(vec=1, rows=1, warps=4, prefetch=1),
    dict(vec=2, rows=2, warps=4, prefetch=1),
]
TUNE_STEPS = 48


def _cache_path():
    p = os.environ.get("TAICHIRTM_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "taichirtm_b200", "autotune.json")


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(cache):
    p = _cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = f"{p}.{os.getpid()}.tmp"  # one per process: ranks may store at the same time
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def key(nz, shots, modes):
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    rows = sum(s.nx for s in shots)
    return f"{name}|nz={nz}|rows={rows}|shots={len(shots)}|modes={modes}|v10"


def time_shape(make_plan, shots, tune, steps=TUNE_STEPS):
    """ms per time step of a forward loop replayed as a CUDA graph (how the
    batched and plain runs execute; direct launches would favour shapes with
    fewer launches on small, launch-bound grids).  Best of two replays."""
    p = make_plan(dict(tune, graphs=1), steps)
    try:
        nsrc = sum(len(s.src) for s in shots)
        wav = torch.zeros((3, nsrc, steps), dtype=torch.float32, device=p.device)
        if nsrc:
            wav[:, :, 1] = 1.0
        p.forward(wav, check_interval=0)  # captures the graph
        torch.cuda.synchronize()
        best = None
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            p.forward(wav, check_interval=0)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            best = ms if best is None else min(best, ms)
        return best
    finally:
        p.close()


def best_shape(make_plan, nz, shots, modes, nt, candidates=None, refresh=False):
    """Cached best launch shape; tunes on a miss."""
    k = key(nz, shots, modes)
    cache = _load()
    if not refresh and k in cache:
        return cache[k]["tune"]
    results = []
    for t in candidates or CANDIDATES:
        try:
            results.append((time_shape(make_plan, shots, t), t))
        except Exception:
            continue
    if not results:
        return None
    ms, best = min(results, key=lambda r: r[0])
    cache[k] = dict(tune=best, ms_per_step=ms, tried=[dict(t, ms=m) for m, t in results])
    _store(cache)
    return best


# FWI gradients: the exact adjoint kernel dominates and prefers more, smaller
# warp tasks than the forward step, so FWIProblem(tune="auto") times the
# gradient itself (checkpointed forward + adjoint sweep) on a short time axis.
FWI_CANDIDATES = ([dict(vec=2, rows=r, warps=w, tsteps=2) for r in (4, 8, 16) for w in (1, 2, 4)]
                  + [dict(vec=2, rows=32, warps=w, tsteps=2) for w in (1, 2)]
                  # 24-row tasks: with the tail split, 1.7 % faster than 16 rows on the c4 gradient
                  + [dict(vec=2, rows=24, warps=w, tsteps=2) for w in (2, 4)]
                  # material ring with the task from the block index for the forward and recompute
                  # launches (one warp per CTA, so the adjoint takes its uniform-task form too)
                  + [dict(vec=2, rows=r, warps=1, tsteps=2, prefetch=4) for r in (8, 16, 32)])
FWI_TUNE_STEPS = 160


def time_fwi_shape(make_problem, nx, nz, tune, steps=FWI_TUNE_STEPS):
    """ms per time step of one gradient (checkpointed forward + adjoint) on a
    homogeneous model; kernel times do not depend on the values."""
    prob = make_problem(tune, steps)
    try:
        dev = prob.device
        rho = torch.full((nx, nz), 2200.0, dtype=torch.float32, device=dev)
        mu = rho * 1400.0 ** 2
        lam = rho * 2500.0 ** 2 - 2 * mu
        seis, ck, _ = prob.forward(lam, mu, rho)
        prob.adjoint(seis, ck)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        seis, ck, _ = prob.forward(lam, mu, rho)
        prob.adjoint(seis, ck)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    finally:
        prob.close()


def best_fwi_shape(make_problem, nx, nz, shots, candidates=None, refresh=False):
    """Cached best launch shape for FWI gradients; tunes on a miss."""
    k = "fwi|" + key(nz, shots, 1)
    cache = _load()
    if not refresh and k in cache:
        return cache[k]["tune"]
    results = []
    for t in candidates or FWI_CANDIDATES:
        try:
            results.append((time_fwi_shape(make_problem, nx, nz, t), t))
        except Exception:
            continue
    if not results:
        return None
    ms, best = min(results, key=lambda r: r[0])
    cache[k] = dict(tune=best, ms_per_step=ms, tried=[dict(t, ms=m) for m, t in results])
    _store(cache)
    return best
