#!/usr/bin/env python
"""Benchmark: batched P-SV reverse-time migration on one B200 (per GPU).

Workload (one "step"): 64 shots of the batched P-SV RTM configuration -- a
2001 x 801 model (dx = 5 m, dt = 0.5 ms, nt = 3000, 4 layers + 20 seeded
anomalies), shot k at x index 55 + 30 k with U{200..800} receivers in a window
+- a 50-cell sponge -- migrated in one pass: forward with snapshots every 16
steps, backward with Kahan zero-lag cross-correlation, FP64 stack of all 64
images on the global grid.  Each kernel launch advances all 64 shots by one
time step, or by two (temporal blocking, when the autotuner picks it).
Observed data are modelled on the true model before timing.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun the job is N copies of the 64-shot survey (weak scaling: 64
shots per GPU); taichirtm_b200.distributed.shard_shots splits them across the
ranks by cost and reduce_result sums the stacked images with one FP64
all-reduce after a status agreement, the shipped sharded path.

Besides the headline line, the default run also times, with their own clock
records, the FWI gradient (8 shots on 1201 x 401, batched against one shot per
problem) and checkpointed RTM (the same 64 shots with sqrt(nt) checkpoints,
batched against one shot per plan): keys "gradient" and "checkpointed_rtm".
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RTM shots/s & Gcell-upd/s, batched vs plain on one B200, at <=1e-4 image err"
ISNAP = 16
STATE_BYTES_PER_CELL = 40    # P-SV: 5 state fields read + written, per shot cell
MATERIAL_BYTES_PER_CELL = 20  # P-SV: 5 material fields read once per model cell (shared by shots)
SNAP_BYTES_PER_CELL = 8      # forward snapshot step: u, w written
IMG_BYTES_PER_CELL = 40      # imaging step: u, w snapshot read (8) + Kahan sum/comp RMW (32)
PEAK_FALLBACK_GBS = 6650.0


def workload_desc(nshots, nt):
    return (f"batched P-SV RTM: {nshots} shots on a 2001x801 model (dx=5 m, dt=0.5 ms, nt={nt}), "
            "windows of U{200..800} receivers +- 50-cell sponge, isnap=16, Kahan imaging, FP64 stack")


def bench_config(nshots, nt, world, cells):
    """The workload as both arms name it (the same dict in both lines)."""
    return dict(workload=workload_desc(nshots, nt), shots_per_gpu=nshots, cells_per_shot_step=int(cells),
                grid="2001x801", nt=nt, isnap=ISNAP,
                l2="no flush: per-step working set (state 2.6 GB + snapshots 48 GB) >> 126 MB L2",
                parallelism=f"{world} x {nshots} shots sharded by cost across {world} GPU(s), "
                            "FP64 all-reduce of the image")


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def ncu_traffic_per_cell(tsteps=1):
    """DRAM bytes per shot cell of ONE launch of the step kernel that runs
    `tsteps` time steps per launch, from the committed ncu summary
    (profiles/step_kernel_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "step_kernel_traffic.json")) as f:
            k = json.load(f)["kernels"][str(int(tsteps))]
        return float(k["dram_bytes_per_shot_cell_per_launch"])
    except Exception:
        return None


def build_workload(nt):
    from taichirtm_b200 import synthetic as S
    return S.config3(nt=nt)


# --------------------------------------------------------------------------- CPU
def cpu_rtm_shot(survey, k, n_run=None, modes=3):
    """The reference algorithm on the host cores (C/OpenMP FP32 restatement of
    src/forward_modeling.py + src/backward_modeling.py, both P-SV and SH as the
    reference always advances): shot k of the workload on its window, forward
    with snapshots every ISNAP steps, backward with imaging.  n_run None = the
    whole time axis.  Returns (seconds, dict describing the run)."""
    from oracle import c_oracle
    sh = survey.shots[k]
    mu, lam, rho = survey.material(migration=True)
    mu, lam, rho = (np.ascontiguousarray(x[sh.x0:sh.x0 + sh.nx]) for x in (mu, lam, rho))
    nthreads = os.cpu_count() or 1
    nt = survey.nt
    n_run = nt if n_run is None else int(min(nt, n_run))
    kw = dict(dx=survey.dx, dz=survey.dz, nt=nt, fs=survey.fs, fw=survey.fw, dtype=np.float32,
              modes=modes, nthreads=nthreads)
    t0 = time.perf_counter()
    f = c_oracle.forward(mu, lam, rho, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2],
                         rec=sh.rec, nt_run=n_run, save=True, isnap=ISNAP, **kw)
    c_oracle.backward(mu, lam, rho, rec=sh.rec, obs=np.zeros((3, len(sh.rec), nt), np.float32),
                      snaps=f["snaps"], isnaps=np.arange(1, nt // ISNAP + 1) * ISNAP,
                      num_snaps=nt // ISNAP, isnap=ISNAP, nt_run=n_run, **kw)
    sec = time.perf_counter() - t0
    return sec, dict(cores=nthreads, kind="port", cells=sh.nx * survey.nz, nx=sh.nx, n_run=n_run)


def cpu_rtm_sample(survey):
    """cpu_baseline leg of the GPU arm: shot 0 migrated in full on the host
    cores (a bounded sample of the workload, about 5 s on 16 cores)."""
    sec, d = cpu_rtm_shot(survey, 0)
    nt = survey.nt
    return dict(value=1.0 / sec, unit="shots/s", cores=d["cores"], kind="port",
                gcell_upd_per_s=2 * d["cells"] * nt / sec / 1e9,
                sample=(f"shot 0 ({d['nx']}x{survey.nz} window), all {nt} steps of both phases "
                        f"(forward with snapshots + backward with imaging), FP32, P-SV+SH as the "
                        f"reference runs"))


def reference_arm(args, rank):
    """The reference's algorithm on the host cores (Taichi cannot be installed
    offline, so the C/OpenMP restatement of its kernels): every step is one
    whole shot of the workload -- shots taken in turn, all nt steps of the
    forward with snapshots and the backward with imaging -- so ms_per_step is
    the measured time of one step and value = timed shots / timed seconds."""
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    survey = build_workload(3000)
    import platform
    times = []
    info = None
    for i in range(args.warmup + args.steps):
        sec, info = cpu_rtm_shot(survey, i % len(survey.shots))
        if i >= args.warmup:
            times.append(sec)
    total = float(sum(times))
    v = args.steps / total
    cells = sum(s.nx for s in survey.shots) * survey.nz
    sample = (f"{args.steps} whole shots (shots {args.warmup % 64}.. in turn, after {args.warmup} untimed), "
              f"all 3000 steps of both phases each, FP32, P-SV+SH as the reference runs, "
              f"{info['cores']} host threads")
    line = dict(impl="reference", metric=METRIC, value=v, unit="shots/s", n_gpus=world,
                steps=args.steps, warmup=args.warmup, ms_per_step=1000.0 * total / args.steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                config=bench_config(64, 3000, world, cells),
                step="one whole shot of the workload on the host cores",
                host=platform.processor() or platform.machine(),
                cpu_baseline=dict(value=v, unit="shots/s", cores=info["cores"], kind="port", sample=sample),
                e2e=dict(value=v, unit="shots/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                note="Taichi (the reference's runtime) is not installable offline; the reference arm "
                     "times the C/OpenMP restatement of its kernels on all host cores")
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ large model (c5)
def c5_host_legs(line):
    """Host legs of the large-model line, on its shot 0 (a 1339 x 1601 window):
    the cpu_baseline (the C restatement in FP32, both P-SV and SH as the
    reference runs, a bounded sample of the time axis scaled to one shot),
    and, as the checker, the FP64 run of the same restatement against which
    the shot's RTM image is compared for snapshots and each checkpoint
    storage (full length; snapshots and imaging every 160 steps to bound the
    host memory of the FP64 snapshots)."""
    import torch
    from oracle import c_oracle
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    sv, K, tune = line["_survey"], line["_K"], line["_tune"]
    sh = sv.shots[0]
    crop = [np.ascontiguousarray(x[sh.x0:sh.x0 + sh.nx]) for x in sv.material(migration=True)]
    nthreads = os.cpu_count() or 1
    n_run = 400
    kw = dict(dx=sv.dx, dz=sv.dz, nt=sv.nt, fs=sv.fs, fw=sv.fw, nthreads=nthreads)
    t0 = time.perf_counter()
    f = c_oracle.forward(*crop, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2], rec=sh.rec,
                         nt_run=n_run, save=True, isnap=ISNAP, dtype=np.float32, modes=3, **kw)
    c_oracle.backward(*crop, rec=sh.rec, obs=np.zeros((3, len(sh.rec), sv.nt), np.float32), snaps=f["snaps"],
                      isnaps=np.arange(1, sv.nt // ISNAP + 1) * ISNAP, num_snaps=sv.nt // ISNAP, isnap=ISNAP,
                      nt_run=n_run, dtype=np.float32, modes=3, **kw)
    sec = (time.perf_counter() - t0) * sv.nt / n_run
    del f
    line["cpu_baseline"] = dict(value=round(1.0 / sec, 5), unit="shots/s (RTM)", cores=nthreads, kind="port",
                                sample=f"shot 0 ({sh.nx}x{sv.nz} window), {n_run} of {sv.nt} steps of both phases, "
                                       f"FP32, P-SV+SH as the reference runs, scaled x{sv.nt // n_run} to one shot")
    ie = 160
    f64 = c_oracle.forward(*crop, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2], rec=sh.rec,
                           save=True, isnap=ie, snap_comps=(0, 2), dtype=np.float64, modes=1, **kw)
    obs = (0.5 * f64["seis"]).astype(np.float32)
    img64 = c_oracle.backward(*crop, rec=sh.rec, obs=obs, snaps=f64["snaps"], isnaps=f64["isnaps"],
                              num_snaps=f64["num_snaps"], isnap=ie, snap_comps=(0, 2), dtype=np.float64, modes=1,
                              **kw)["img"]
    del f64
    r = BatchedRTM(*sv.material(migration=True), sv.dx, sv.dz, sv.fs, sv.nt, sv.fw,
                   [ShotGeometry(sh.x0, sh.nx, sh.src, sh.rec)], tune=tune, graphs=False)
    errs = {}
    for dt in (None, "f32", "f16", "i16"):
        ck = dict(every=K, dtype=dt) if dt else None
        _, _, st = r.migrate(sh.wavelets, obs, isnap=ie, checkpoint=ck)
        img = st.cpu().numpy()[:, sh.x0:sh.x0 + sh.nx]
        a, b = img[[0, 2]].astype(np.float64), img64[[0, 2]]
        errs[f"image_{dt or 'snapshots'}_vs_fp64_rel_l2"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    r.close()
    torch.cuda.synchronize()
    line["errors_vs_fp64"] = dict(errs, case=f"shot 0 ({sh.nx}x{sv.nz} window), all {sv.nt} steps, imaging every "
                                             f"{ie} steps, observed data = half the FP64 seismograms; "
                                             "the FP64 C restatement as the checker")


# ------------------------------------------------------------- plain one-shot RTM
def plain_single_shot(args, rank):
    """Plain single-shot RTM (forward with snapshots at the reference's
    interval, backward with imaging) on the full model: 301 x 151 P-SV (c1) or
    1001 x 501 SH (c2), the CPU restatement timed beside it."""
    if rank != 0:
        return 0
    import torch
    from taichirtm_b200 import autotune, synthetic as S
    from taichirtm_b200.benchmarks import ClockSampler
    from taichirtm_b200.plan import PSV, SH, Plan, ShotGeometry
    from oracle import c_oracle
    cfg = S.config1() if args.workload == "c1" else S.config2()
    modes, isnap = (PSV, 1) if args.workload == "c1" else (SH, 7)
    sh = cfg.shots[0]
    geo = [ShotGeometry(0, cfg.nx, sh.src, sh.rec)]
    mk = lambda tune, nt: Plan(cfg.nx, cfg.nz, cfg.dx, cfg.dz, nt, cfg.fs, cfg.fw, modes, geo, tune=tune)  # noqa: E731

    def make(tune, nt):
        p = mk(tune, nt)
        p.set_model(*cfg.material(migration=True))
        return p
    tune = dict(autotune.best_shape(make, cfg.nz, geo, modes, cfg.nt) or {}, graphs=1)
    true = mk(tune, cfg.nt)
    true.set_model(*cfg.material())
    wav = torch.as_tensor(sh.wavelets).cuda()
    _, obs, _, _ = true.forward(wav)
    obs = obs.clone()
    true.close()
    p = make(tune, cfg.nt)
    nsnap = cfg.nt // isnap
    snaps = [p.snapshot_buffer(nsnap) if (c == 1) == (modes == SH) else None for c in range(3)]

    def rtm():
        f1, _, sn, isn = p.forward(wav, save=True, isnap=isnap, snaps=snaps)
        f2, img, _ = p.backward(obs, sn, isn, len(isn), isnap)
        return f1, f2, img
    for _ in range(max(3, args.warmup)):
        f1, f2, img = rtm()
    assert int(f1.max()) == 0 and int(f2.max()) == 0
    torch.cuda.synchronize()
    clk = ClockSampler().start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        rtm()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    cells = cfg.nx * cfg.nz
    # both modes advanced, as the reference always does (the skipped mode is
    # all zeros here, so the images are the same; this is its cost)
    pb = Plan(cfg.nx, cfg.nz, cfg.dx, cfg.dz, cfg.nt, cfg.fs, cfg.fw, PSV | SH, geo, tune=tune)
    pb.set_model(*cfg.material(migration=True))
    snaps_b = [pb.snapshot_buffer(nsnap) for _ in range(3)]

    def rtm_both():
        _, _, sn, isn = pb.forward(wav, save=True, isnap=isnap, snaps=snaps_b)
        pb.backward(obs, sn, isn, len(isn), isnap)
    for _ in range(2):
        rtm_both()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        rtm_both()
    e1.record()
    torch.cuda.synchronize()
    ms_both = e0.elapsed_time(e1) / args.steps
    pb.close()
    del snaps_b
    # CPU: the reference algorithm (both modes, as the reference advances) on all host cores
    mu, lam, rho = cfg.material(migration=True)
    nthreads = os.cpu_count() or 1
    n_run = min(cfg.nt, 400 if args.workload == "c1" else 100)
    kw = dict(dx=cfg.dx, dz=cfg.dz, nt=cfg.nt, fs=cfg.fs, fw=cfg.fw, dtype=np.float32, modes=3, nthreads=nthreads)
    t0 = time.perf_counter()
    f = c_oracle.forward(mu, lam, rho, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2],
                         rec=sh.rec, nt_run=n_run, save=True, isnap=isnap, **kw)
    c_oracle.backward(mu, lam, rho, rec=sh.rec, obs=np.zeros((3, len(sh.rec), cfg.nt), np.float32),
                      snaps=f["snaps"], isnaps=f["isnaps"], num_snaps=f["num_snaps"], isnap=isnap, nt_run=n_run, **kw)
    cpu_s = (time.perf_counter() - t0) * cfg.nt / n_run
    line = dict(metric=METRIC, value=round(1000.0 / ms, 3), unit="shots/s", n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(ms, 3), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f32", data="synthetic",
                config=dict(workload=cfg.name + f": {cfg.nx}x{cfg.nz}, nt={cfg.nt}, isnap={isnap}, one shot, "
                            "forward with snapshots + backward with imaging"),
                launch_shape=tune, clocks=clocks, gcell_upd_per_s=round(2 * cells * cfg.nt / (ms / 1000.0) / 1e9, 2),
                us_per_step=round(ms * 1000.0 / (2 * cfg.nt), 2),
                both_modes=dict(shots_per_s=round(1000.0 / ms_both, 3),
                                note="P-SV and SH both advanced, as the reference does"),
                cpu_baseline=dict(value=round(1.0 / cpu_s, 4), unit="shots/s", cores=nthreads, kind="port",
                                  sample=f"{n_run} of {cfg.nt} steps per phase, both P-SV and SH, FP32, scaled"))
    print(json.dumps(line), flush=True)
    p.close()
    return 0


# --------------------------------------------------------------------------- GPU
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nt", type=int, default=None, help="time steps (default: the workload's)")
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the one-shot-per-launch leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the checkpointed-RTM and FWI-gradient legs of the default workload")
    ap.add_argument("--ckpt-dtype", default=None, choices=["f32", "f16", "bf16", "i16"],
                    help="checkpoint storage of the checkpointed-RTM leg and of c5 (default i16: 16-bit block "
                         "floating point, one scale per 60-column block)")
    ap.add_argument("--tune", default=None,
                    help='fixed launch shape as JSON, e.g. \'{"vec": 2, "rows": 32, "warps": 1, "tsteps": 2}\' '
                         "(default: the autotuner's choice)")
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c3: batched P-SV RTM (default, the headline); c4: FWI gradient, 8 shots "
                         "1201x401; c5: large checkpointed RTM + gradient, 32 shots 4001x1601")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if args.workload in ("c1", "c2"):
        return plain_single_shot(args, rank)
    if args.workload == "c5":
        from taichirtm_b200 import benchmarks
        import torch
        torch.cuda.set_device(local)
        line = benchmarks.run_c5(args)
        if not args.no_cpu:
            c5_host_legs(line)
        for k in [k for k in line if k.startswith("_")]:
            line.pop(k)
        print(json.dumps(line), flush=True)
        return 0
    if args.workload != "c3":
        from taichirtm_b200 import benchmarks
        return benchmarks.run(args)

    import torch
    import torch.distributed as dist
    from taichirtm_b200.batch import BatchedRTM, survey_shots
    from taichirtm_b200.benchmarks import ClockSampler
    from taichirtm_b200.distributed import reduce_result, shard_shots
    from taichirtm_b200.plan import PSV

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    survey = build_workload(args.nt or 3000)
    survey.shots = survey.shots[: args.shots]
    # the job: `world` copies of the survey's shots, split across the ranks by
    # cost (window cells) -- each rank gets one copy of every shot
    base = survey.shots
    job = [k for _ in range(world) for k in range(len(base))]
    mine = shard_shots([base[k].nx * survey.nz for k in job], world, rank)
    survey.shots = [base[job[i]] for i in mine]
    shots = survey_shots(survey)
    wav = torch.as_tensor(np.concatenate([s.wavelets for s in survey.shots], axis=1)).to(dev)
    mu_t, lam_t, rho_t = survey.material()
    mu_m, lam_m, rho_m = survey.material(migration=True)

    # observed data: forward on the true model (untimed)
    true = BatchedRTM(mu_t, lam_t, rho_t, survey.dx, survey.dz, survey.fs, survey.nt, survey.fw, shots,
                      modes=PSV, tune=json.loads(args.tune) if args.tune else "auto", device=dev)
    flags, obs, _, _ = true.forward(wav, save=False, check_interval=100)
    assert int(flags.max()) == 0, flags
    obs = obs.clone()
    true.close()
    del true
    rtm = BatchedRTM(mu_m, lam_m, rho_m, survey.dx, survey.dz, survey.fs, survey.nt, survey.fw, shots,
                     modes=PSV, tune=json.loads(args.tune) if args.tune else "auto", device=dev)
    plan = rtm.plan
    cells = rtm.cells()
    nt = survey.nt
    nsnap = nt // ISNAP
    n_img = sum(1 for t in range(1, nt) if t % ISNAP == 0 and t // ISNAP - 1 < nsnap)
    stack = torch.zeros((3, survey.nx, survey.nz), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def one_step(ev=None):
        if ev:
            ev[0].record(stream)
        ff, _, snaps, isnaps = plan.forward(wav, save=True, isnap=ISNAP, check_interval=100)
        n_launch = plan.launch_count()  # step launches + seismogram transpose
        if ev:
            ev[1].record(stream)
        fb, _, _ = plan.backward(obs, snaps, isnaps, len(isnaps), ISNAP, check_interval=100, image=False,
                                 stack=stack)
        n_launch += plan.launch_count()  # transpose + step launches + stack
        if ev:
            ev[2].record(stream)
        return ff, fb, n_launch

    status = 0
    for _ in range(args.warmup):
        ff, fb, _ = one_step()
        status = max(status, int(ff.max()), int(fb.max()))
    torch.cuda.synchronize()
    if world > 1:
        reduce_result(torch.zeros(1, dtype=torch.float64, device=dev), status)  # all ranks agree or raise
    elif status:
        raise FloatingPointError(f"propagation became non-finite (code {status})")
    sampler = ClockSampler().start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    launches = 0
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier(device_ids=[local])
    t_start.record(stream)
    for k in range(args.steps):
        ff, fb, n_launch = one_step(evs[k])
        status = max(status, int(ff.max()), int(fb.max()))
        launches += n_launch
    if world > 1:
        stack = reduce_result(stack, status)  # cross-GPU image stack (FP64), after a status check
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier(device_ids=[local])
    clocks = sampler.stop()
    ms = t_start.elapsed_time(t_end)
    fwd_ms = sum(e[0].elapsed_time(e[1]) for e in evs)
    bwd_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    n_job = torch.tensor([len(shots)], device=dev)
    if world > 1:
        dist.all_reduce(n_job, op=dist.ReduceOp.SUM)
    shots_total = int(n_job.item()) * args.steps
    value = shots_total / (ms / 1000.0)
    gcell = 2.0 * cells * nt * world * args.steps / (ms / 1000.0) / 1e9

    # roofline of the fused step kernels (forward + backward launches of the timed
    # region).  Compulsory bytes per step, the batched form of the per-cell
    # figure: every shot's state read and written once (40 B per shot cell) and
    # the shared material read once per model cell covered by any window
    # (20 B per union cell); plus snapshot writes / imaging reads+RMW.
    covered = np.zeros(survey.nx, bool)
    for s_ in shots:
        covered[s_.x0:s_.x0 + s_.nx] = True
    union_cells = int(covered.sum()) * survey.nz
    step_bytes = STATE_BYTES_PER_CELL * cells + MATERIAL_BYTES_PER_CELL * union_cells
    n_snap_writes = nsnap if nsnap * ISNAP <= nt - 1 else nsnap - 1
    alg_fwd = nt * step_bytes + n_snap_writes * SNAP_BYTES_PER_CELL * cells
    alg_bwd = nt * step_bytes + n_img * IMG_BYTES_PER_CELL * cells
    # per time step (the unit of the byte model); a launch runs tsteps steps
    tsteps = int(rtm.tune.get("tsteps", 1) or 1)
    per_step_bytes = (alg_fwd + alg_bwd) / (2 * nt)
    per_step_ms = (fwd_ms + bwd_ms) / args.steps / (2 * nt)
    achieved = per_step_bytes / (per_step_ms * 1e-3) / 1e9
    peak, peak_kind = peak_hbm()
    tpc = ncu_traffic_per_cell(tsteps)
    roofline = dict(bound="hbm", achieved=round(achieved, 1), peak=peak, unit="GB/s",
                    frac=round(achieved / peak, 4),
                    traffic=(round(tpc * cells) if tpc else None),
                    kernel=(f"step2_kernel<fwd|bwd, P-SV>: one launch = {tsteps} time steps of all shots"
                            if tsteps == 2 else "step_kernel<fwd|bwd, P-SV>: one launch = one time step of all shots"),
                    steps_per_launch=tsteps,
                    bytes_per_launch=int(per_step_bytes * tsteps), us_per_launch=round(per_step_ms * tsteps * 1e3, 2),
                    bytes_model=("algorithmic bytes per time step: 40 B per shot cell (state R+W) + 20 B per "
                                 "model cell under any window (material read once) + snapshot / imaging bytes; "
                                 "x steps per launch. traffic = ncu DRAM bytes of one launch"),
                    achieved_if_material_per_shot=round(
                        (per_step_bytes + MATERIAL_BYTES_PER_CELL * (cells - union_cells)) / (per_step_ms * 1e-3) / 1e9, 1),
                    peak_source=peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind)
    if tpc:
        dram_gbs = tpc * cells / (per_step_ms * tsteps * 1e-3) / 1e9
        roofline["dram_achieved"] = round(dram_gbs, 1)
        roofline["dram_frac"] = round(dram_gbs / peak, 4)

    # end to end through the public API: host inputs, device outputs read back
    # into pinned host memory every step
    wav_h = wav.cpu().pin_memory()
    obs_h = obs.cpu().pin_memory()
    host_img = torch.empty(tuple(stack.shape), dtype=stack.dtype).pin_memory()
    h2d = wav_h.numel() * 4 + obs_h.numel() * 4
    d2h = host_img.numel() * 8

    def e2e_step():
        # observed data stay in pinned host memory: migrate copies them on a
        # side stream while the forward pass runs (the backward reads them)
        ff, fb, st = rtm.migrate(wav_h.to(dev, non_blocking=True), obs_h, isnap=ISNAP, check_interval=100)
        if world > 1:
            st = reduce_result(st, max(int(ff.max()), int(fb.max())))
        host_img.copy_(st, non_blocking=True)
        torch.cuda.current_stream().synchronize()  # the step's image is on the host

    e2e_step()  # warm-up: the side stream's copy buffer is allocated here, not in the timed loop
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = dict(value=shots_total / (e2e_ms / 1000.0), unit="shots/s", h2d_bytes_per_step=int(h2d),
               d2h_bytes_per_step=int(d2h), api="taichirtm_b200.batch.BatchedRTM.migrate")
    assert np.isfinite(host_img.numpy()).all()

    def plain_rate(nplain, checkpoint=None):
        """The plain path: shots 0 .. nplain-1 migrated one shot per plan (one
        shot per launch), same semantics, each plan with its own autotuned
        launch shape; each timed once after one untimed call."""
        t_sum, shapes = 0.0, []
        for s in range(nplain):
            sub = [shots[s]]
            o0 = sum(len(x.src) for x in shots[:s])
            r0 = sum(len(x.rec) for x in shots[:s])
            one = BatchedRTM(mu_m, lam_m, rho_m, survey.dx, survey.dz, survey.fs, nt, survey.fw, sub,
                             modes=PSV, tune="auto", device=dev)  # each one-shot plan tuned for itself
            shapes.append({k: v for k, v in one.tune.items() if k != "graphs"})
            w1 = wav[:, o0:o0 + len(sub[0].src)].contiguous()
            o1 = obs[:, r0:r0 + len(sub[0].rec)].contiguous()
            one.migrate(w1, o1, isnap=ISNAP, checkpoint=checkpoint)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one.migrate(w1, o1, isnap=ISNAP, checkpoint=checkpoint)
            b.record(stream)
            torch.cuda.synchronize()
            t_sum += a.elapsed_time(b)
            one.close()
        return dict(shots_per_s=round(nplain / (t_sum / 1000.0), 3), launch_shapes=shapes,
                    sample=f"shots 0..{nplain - 1} migrated one shot per plan (one shot per launch), "
                           "each plan with its own autotuned launch shape")

    # the plain path, checkpointed RTM and gradient legs are one-GPU
    # comparisons: run at N = 1 only, so an N-GPU run holds its GPUs for the
    # sharded headline alone
    plain = None
    if not args.no_plain and world == 1:
        plain = plain_rate(4)

    # checkpointed RTM: the same shots with sqrt(nt) checkpoints and the
    # forward wavefield recomputed segment by segment, batched vs plain
    ckpt_rtm = None
    if not args.no_extra and world == 1:
        ck = dict(every=max(1, round(nt ** 0.5)), dtype=args.ckpt_dtype or "i16")
        rtm.migrate(wav, obs, isnap=ISNAP, checkpoint=ck)
        torch.cuda.synchronize()
        clk = ClockSampler().start()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(2):
            ffc, fbc, _ = rtm.migrate(wav, obs, isnap=ISNAP, checkpoint=ck)
        b.record(stream)
        torch.cuda.synchronize()
        cclk = clk.stop()
        assert int(ffc.max()) == 0 and int(fbc.max()) == 0
        c_ms = a.elapsed_time(b) / 2
        c_rate = len(shots) / (c_ms / 1000.0)
        c_plain = plain_rate(4, checkpoint=ck)
        ckpt_rtm = dict(shots_per_s=round(c_rate, 3), ms_per_step=round(c_ms, 2), steps=2, warmup=1,
                        checkpoint=ck, clocks=cclk, plain=c_plain,
                        batched_vs_plain=round(c_rate / c_plain["shots_per_s"], 2),
                        workload=workload_desc(len(shots), nt) + f", checkpoints every {ck['every']} steps "
                                 f"({ck['dtype']}) with recompute instead of snapshots")

    gradient = None
    if not args.no_extra and world == 1:
        from taichirtm_b200 import benchmarks
        gradient = benchmarks.gradient_leg(nt=3000, steps=3, warmup=1, nplain=2)

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_rtm_sample(survey)

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = dict(
            metric=METRIC, value=round(value, 4), unit="shots/s", n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=round(ms_per_step, 2), higher_is_better=True, scaling="weak",
            vs_baseline=None, dtype="f32", data="synthetic",
            config=bench_config(len(base), nt, world, cells), launch_shape=rtm.tune,
            gcell_upd_per_s=round(gcell, 2), roofline=roofline, e2e=e2e,
            gpu_launches=int(launches), clocks=clocks, cpu_baseline=cpu)
        if plain:
            line["plain"] = plain
            line["batched_vs_plain"] = round(value / world / plain["shots_per_s"], 2)
        if ckpt_rtm:
            line["checkpointed_rtm"] = ckpt_rtm
        if gradient:
            line["gradient"] = gradient
        print(json.dumps(line), flush=True)
    rtm.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
