"""Runners for the FWI-gradient and large checkpointed workloads
(``python bench.py --workload c4|c5``); the default ``bench.py`` workload is
the batched P-SV RTM.  Each prints one JSON line.

c4  FWI gradient: 1201 x 401 model, dx = 5 m, dt = 0.5 ms, nt = 3000, 8
    full-spread shots; observed data on the true model, gradient of the L2
    misfit on vx and vz w.r.t. (vp, vs, rho) at the Gaussian-smoothed
    (sigma 15 cells) starting model, sqrt(nt) FP32 checkpoints with recompute.
c5  Large batched, checkpointed P-SV RTM plus gradient: 4001 x 1601, dt =
    0.4 ms, nt = 8000, 32 shots with U{1000..2000} receivers, FP16
    per-field-scaled checkpoints, shots processed in waves that fit HBM.
"""
import json
import math
import os
import subprocess
import tempfile

import numpy as np
import torch

from . import synthetic as S
from .batch import BatchedRTM, survey_shots, survey_wavelets
from .fwi import FWIProblem, l2_misfit
from .plan import PSV


def _ev():
    return torch.cuda.Event(enable_timing=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while a
    timed region runs (start before it, stop after it)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def stop(self, gpu_index=None):
        """dict(sm_mhz = median under load, sm_max_mhz, reasons, samples), or
        None without nvidia-smi.  gpu_index defaults to the first entry of
        CUDA_VISIBLE_DEVICES."""
        if self.p is None:
            return None
        if gpu_index is None:
            gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0] or None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if gpu_index is not None:
            sel = [r for r in rows if r[0].strip() == str(gpu_index)]
            rows = sel or rows
        if not rows:
            return None
        sm = np.array([float(r[1]) for r in rows])
        mx = max(float(r[2]) for r in rows)
        pw = np.array([float(r[3]) if r[3].strip() not in ("[N/A]", "N/A") else 0 for r in rows])
        load = sm[pw > 0.5 * pw.max()] if pw.max() > 0 else sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return dict(sm_mhz=float(np.median(load)), sm_max_mhz=mx, reasons=reasons, samples=len(rows))


_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PEAK_FALLBACK_GBS = 6650.0
STATE_BYTES_PER_CELL = 40     # P-SV state read + written once per time step, per shot cell
MATERIAL_BYTES_PER_CELL = 20  # P-SV material read once per time step, per model cell under any window
KAHAN_IMG_BYTES_PER_CELL = 32  # imaging step: Kahan sum/compensation RMW of u and w


def _peak_hbm():
    try:
        with open(os.path.join(_ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def _union_cells(shots, nz):
    rows = set()
    for s in shots:
        rows.update(range(s.x0, s.x0 + s.nx))
    return len(rows) * nz


def _step_bytes(shots, nz):
    """Compulsory bytes of one P-SV time step of one phase for a batch: every
    shot's state read and written once, the shared material read once."""
    return STATE_BYTES_PER_CELL * sum(s.nx for s in shots) * nz + MATERIAL_BYTES_PER_CELL * _union_cells(shots, nz)


def _roofline(nbytes, ms, model):
    peak, kind = _peak_hbm()
    achieved = nbytes / (ms / 1000.0) / 1e9
    return dict(bound="hbm", achieved=round(achieved, 1), peak=peak, unit="GB/s", frac=round(achieved / peak, 4),
                traffic=None, bytes_model=model, algorithmic_bytes=int(nbytes),
                peak_source=kind + (" (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else ""))


def _corr(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-300))


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300))


def _plain_gradient(sv, shots, wav, obs, m0, K, nt, dev, nplain):
    """The same gradient, one shot per problem (one shot per launch), each
    problem with its own autotuned launch shape: shots/s over shots
    0 .. nplain-1, each timed once after one untimed call."""
    t_sum, shapes = 0.0, []
    for s in range(nplain):
        o0 = sum(len(x.src) for x in shots[:s])
        r0 = sum(len(x.rec) for x in shots[:s])
        w1 = wav[:, o0:o0 + len(shots[s].src)].contiguous()
        ob1 = obs[:, r0:r0 + len(shots[s].rec)].contiguous()
        one = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, nt, sv.fw, [shots[s]], w1, ckpt_every=K,
                         tune="auto", device=dev)
        shapes.append(one.tune)

        def grad1():
            m = [x.clone().requires_grad_(True) for x in m0]
            l2_misfit(m[0], m[1], m[2], one, ob1).backward()
        grad1()
        torch.cuda.synchronize()
        a, b = _ev(), _ev()
        a.record()
        grad1()
        b.record()
        torch.cuda.synchronize()
        t_sum += a.elapsed_time(b)
        one.close()
    return dict(shots_per_s=round(nplain / (t_sum / 1000.0), 3), launch_shapes=shapes,
                sample=f"shots 0..{nplain - 1}, one shot per problem (one shot per launch), "
                       "each with its own autotuned launch shape")


def gradient_leg(nt=3000, steps=3, warmup=1, nplain=2, with_reference_image=False):
    """The c4 FWI gradient, timed: 8 shots on the 1201 x 401 model in one
    problem (every launch advances all shots) against the same gradient one
    shot per problem (the plain path).  Returns a dict with the batched
    gradient shots/s, its roofline in compulsory bytes, the plain figure and
    the clocks of the timed region."""
    sv = S.config4(nt=nt)
    dev = torch.device("cuda")
    shots = survey_shots(sv)
    wav = torch.as_tensor(survey_wavelets(sv), device=dev)
    true = BatchedRTM(*sv.material(), sv.dx, sv.dz, sv.fs, nt, sv.fw, shots, tune="auto", device=dev)
    f, obs, _, _ = true.forward(wav)
    assert int(f.max()) == 0
    obs = obs.clone()
    tune = true.tune
    true.close()
    K = max(1, round(math.sqrt(nt)))
    prob = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, nt, sv.fw, shots, wav, ckpt_every=K,
                      tune="auto", device=dev)
    m0 = [torch.tensor(x, dtype=torch.float64, device=dev) for x in (sv.vp_mig, sv.vs_mig, sv.rho_mig)]

    def gradient():
        m = [x.clone().requires_grad_(True) for x in m0]
        J = l2_misfit(m[0], m[1], m[2], prob, obs)
        J.backward()
        return float(J), [x.grad for x in m]

    for _ in range(max(1, warmup)):
        J, g = gradient()
    torch.cuda.synchronize()
    clk = ClockSampler().start()
    e0, e1 = _ev(), _ev()
    e0.record()
    for _ in range(steps):
        J, g = gradient()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / steps
    cells = sum(s.nx for s in shots) * sv.nz
    plain = _plain_gradient(sv, shots, wav, obs, m0, K, nt, dev, nplain=nplain)
    grad_bytes = 2 * nt * _step_bytes(shots, sv.nz) + 2 * prob.checkpoint_bytes()
    roof = _roofline(grad_bytes, ms, "whole gradient of all shots: 2 phases x nt x (40 B per shot cell + 20 B per "
                                     "model cell under any window) + checkpoints written and read once; the "
                                     "recompute and the gradient sums are not counted; timed end to end per gradient")
    out = dict(shots_per_s=round(len(shots) / (ms / 1000.0), 3), ms_per_gradient=round(ms, 2),
               gcell_upd_per_s=round(2 * cells * nt / (ms / 1000.0) / 1e9, 2), roofline=roof, misfit=J,
               plain=plain, batched_vs_plain=round(len(shots) / (ms / 1000.0) / plain["shots_per_s"], 2),
               clocks=clocks, steps=steps, warmup=max(1, warmup), ckpt_every=K,
               checkpoint_gb=round(prob.checkpoint_bytes() / 1e9, 2),
               launch_shape=dict(rtm=tune, gradient=prob.tune),
               workload=("c4 FWI gradient: 8 shots, 1201x401, dx=5 m, dt=0.5 ms, "
                         f"nt={nt}, L2 misfit on vx and vz, start = smoothed true model (sigma 15), "
                         f"sqrt(nt) = {K}-step FP32 checkpoints with recompute"))
    prob.close()
    if with_reference_image:
        # reference backward + imaging (zero-lag cross-correlation) with the data
        # residual as "observed data": its image vs the exact gradient (reported)
        rtm = BatchedRTM(*sv.material(migration=True), sv.dx, sv.dz, sv.fs, nt, sv.fw, shots,
                         tune={k: v for k, v in tune.items() if k != "graphs"}, graphs=False, device=dev)
        _, syn, _, _ = rtm.forward(wav)
        resid = (syn - obs).contiguous()
        _, _, img = rtm.migrate(wav, resid, isnap=5)
        rtm.close()
        img = img.cpu().numpy()
        inner = (slice(sv.fw, sv.nx - sv.fw), slice(5, sv.nz - sv.fw))
        image_pm = img[0] + img[2]
        out["normalized_corr_gradient_vs_reference_rtm_image"] = {
            k: _corr(gk.cpu().numpy()[inner], image_pm[inner]) for k, gk in zip(("vp", "vs", "rho"), g)}
    return out


def run_c4(args):
    nt = args.nt or 3000
    r = gradient_leg(nt=nt, steps=args.steps, warmup=args.warmup, with_reference_image=True)
    line = dict(metric="FWI gradient shots/s (P-SV, exact adjoint, sqrt(nt) FP32 checkpoints)",
                value=r["shots_per_s"], unit="shots/s", n_gpus=1, steps=args.steps,
                warmup=r["warmup"], ms_per_step=r["ms_per_gradient"], higher_is_better=True, dtype="f32",
                data="synthetic", config=dict(workload=r["workload"], ckpt_every=r["ckpt_every"],
                                               checkpoint_gb=r["checkpoint_gb"]),
                launch_shape=r["launch_shape"], gcell_upd_per_s=r["gcell_upd_per_s"], roofline=r["roofline"],
                misfit=r["misfit"], plain=r["plain"], batched_vs_plain=r["batched_vs_plain"], clocks=r["clocks"],
                normalized_corr_gradient_vs_reference_rtm_image=r["normalized_corr_gradient_vs_reference_rtm_image"],
                note="finite-difference (FP64) and dot-product checks: tests/test_gpu_adjoint.py, "
                     "tests/test_gpu_configs_fp64.py")
    print(json.dumps(line), flush=True)
    return 0


def run_c5(args):
    """The large-model workload: all 32 shots in waves that fit HBM, each wave
    migrated (checkpointed RTM) and differentiated (FWI gradient) in one plan,
    checkpoints in args.ckpt_dtype (default int16 block floating point).
    Returns the JSON line (dict); keys starting with "_" carry the survey and
    shapes for bench.py's host legs and are not printed."""
    nt = args.nt or 8000
    sv = S.config5(nt=nt)
    dev = torch.device("cuda")
    wave = args.shots if args.shots != 64 else 16
    K = max(1, round(math.sqrt(nt)))
    isnap = 16
    cdt = getattr(args, "ckpt_dtype", None) or "i16"
    all_shots = survey_shots(sv)
    all_wav = survey_wavelets(sv)
    t_true = sv.material()
    t_mig = sv.material(migration=True)
    stack = torch.zeros((3, sv.nx, sv.nz), dtype=torch.float64, device=dev)
    grad = None
    t_rtm = t_grad = 0.0
    rtm_bytes = grad_bytes = 0
    peak_mem = 0
    errs = {}
    tune = None
    clk = ClockSampler().start()
    for w0 in range(0, len(all_shots), wave):
        sl = slice(w0, w0 + wave)
        shots = all_shots[sl]
        wav = torch.as_tensor(all_wav[:, sl], device=dev)
        tr = BatchedRTM(*t_true, sv.dx, sv.dz, sv.fs, nt, sv.fw, shots, tune=tune or "auto", graphs=False, device=dev)
        tune = {k: v for k, v in tr.tune.items() if k != "graphs"}
        f, obs, _, _ = tr.forward(wav)
        assert int(f.max()) == 0
        obs = obs.clone()
        tr.close()
        rtm = BatchedRTM(*t_mig, sv.dx, sv.dz, sv.fs, nt, sv.fw, shots, tune=tune, graphs=False, device=dev)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        a, b = _ev(), _ev()
        a.record()
        ff, fb, stack = rtm.migrate(wav, obs, isnap=isnap, stack=stack, checkpoint=dict(every=K, dtype=cdt))
        b.record()
        torch.cuda.synchronize()
        t_rtm += a.elapsed_time(b)
        assert int(ff.max()) == 0 and int(fb.max()) == 0
        shot_cells = sum(s.nx for s in shots) * sv.nz
        n_img = sum(1 for t in range(1, nt) if t % isnap == 0 and t // isnap - 1 < nt // isnap)
        ck_bytes = rtm.checkpoint_bytes(K, cdt)
        rtm_bytes += 2 * nt * _step_bytes(shots, sv.nz) + 2 * ck_bytes + n_img * KAHAN_IMG_BYTES_PER_CELL * shot_cells
        _, syn, _, _ = rtm.forward(wav)
        resid = (syn - obs)
        rtm.close()
        prob = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, nt, sv.fw, shots, wav, ckpt_every=K,
                          ckpt_dtype=cdt, tune="auto", device=dev)
        lam, mu, rho = (torch.as_tensor(x, device=dev) for x in (t_mig[1], t_mig[0], t_mig[2]))
        a.record()
        d, ck, fl = prob.forward(lam, mu, rho)
        g, _ = prob.adjoint(resid, ck)
        b.record()
        torch.cuda.synchronize()
        t_grad += a.elapsed_time(b)
        grad_bytes += 2 * nt * _step_bytes(shots, sv.nz) + 2 * prob.checkpoint_bytes()
        grad_tune = prob.tune
        grad = g if grad is None else grad + g
        del ck
        prob.close()
        peak_mem = max(peak_mem, torch.cuda.max_memory_allocated())
        if w0 == 0:
            # 16-bit checkpoints against FP32 ones at full size, 4-shot subset
            sub = shots[:4]
            ws = wav[:, :4].contiguous()
            nrec = sum(len(s.rec) for s in sub)
            ob = obs[:, :nrec].contiguous()
            rs = resid[:, :nrec].contiguous()
            r2 = BatchedRTM(*t_mig, sv.dx, sv.dz, sv.fs, nt, sv.fw, sub, tune=tune, graphs=False, device=dev)
            imgs = {dt: r2.migrate(ws, ob, isnap=isnap, checkpoint=dict(every=K, dtype=dt))[2].cpu().numpy()
                    for dt in ("f32", "f16", "i16")}
            r2.close()
            gg = {}
            for dt in ("f32", "f16", "i16"):
                pr = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, nt, sv.fw, sub, ws, ckpt_every=K, ckpt_dtype=dt,
                                tune=tune, device=dev)
                d2, c2, _ = pr.forward(lam, mu, rho)
                gg[dt] = pr.adjoint(rs, c2)[0].cpu().numpy()
                del c2
                pr.close()
            for dt in ("f16", "i16"):
                errs[f"image_{dt}_vs_f32_ckpt_rel_l2"] = _rel(imgs[dt][[0, 2]], imgs["f32"][[0, 2]])
                errs[f"gradient_{dt}_vs_f32_ckpt_rel_l2"] = _rel(gg[dt], gg["f32"])
    clocks = clk.stop()
    cells = sum(s.nx for s in all_shots) * sv.nz
    n = len(all_shots)
    return dict(metric="large checkpointed P-SV RTM + FWI gradient shots/s", value=round(n / ((t_rtm + t_grad) / 1000), 4),
                unit="shots/s", n_gpus=1, steps=1, warmup=0, ms_per_step=round(t_rtm + t_grad, 1),
                higher_is_better=True, dtype=f"f32 stencils, {cdt} checkpoints", data="synthetic",
                config=dict(workload=f"c5: {n} shots, 4001x1601, dx=5 m, dt=0.4 ms, nt={nt}, U{{1000..2000}} receivers, "
                                     f"waves of {wave} shots, {cdt} checkpoints (one exponent per 60-column block) "
                                     f"every {K} steps, isnap={isnap}, Kahan images/gradients, FP64 cross-shot sums"),
                launch_shape=dict(rtm=tune, gradient=grad_tune), clocks=clocks,
                rtm_shots_per_s=round(n / (t_rtm / 1000), 4), gradient_shots_per_s=round(n / (t_grad / 1000), 4),
                rtm_gcell_upd_per_s=round(2 * cells * nt / (t_rtm / 1000) / 1e9, 2),
                roofline=dict(rtm=_roofline(rtm_bytes, t_rtm, "checkpointed RTM of all waves: 2 phases x nt x (40 B per "
                                                                "shot cell + 20 B per model cell under any window) + "
                                                                "checkpoints written and read once + 32 B per shot cell per "
                                                                "imaging step (Kahan image RMW); recompute not counted"),
                              gradient=_roofline(grad_bytes, t_grad, "gradient of all waves: 2 phases x nt x (40 B per "
                                                                      "shot cell + 20 B per model cell under any window) "
                                                                      "+ checkpoints written and read once; recompute and "
                                                                      "gradient sums not counted")),
                peak_device_memory_gb=round(peak_mem / 1e9, 1), errors=errs,
                stack_finite=bool(torch.isfinite(stack).all()), grad_finite=bool(torch.isfinite(grad).all()),
                _survey=sv, _tune=tune, _K=K)


def run(args):
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if args.workload == "c4":
        return run_c4(args)
    line = run_c5(args)
    for k in [k for k in line if k.startswith("_")]:
        line.pop(k)
    print(json.dumps(line), flush=True)
    return 0
