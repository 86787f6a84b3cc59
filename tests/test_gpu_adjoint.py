"""GPU checks of the exact discrete adjoint (FWI gradients) and of batched
windowed shots.

* dot-product test of the wavelet adjoint: <F w, g> = <w, F^T g>;
* dot-product test in model space: <J dm, g> (FP64 centred differences of the
  C restatement) = <dm, J^T g> (GPU adjoint) for a random cotangent g;
* gradient w.r.t. (vp, vs, rho) against centred finite differences of the
  SAME discrete forward evaluated in FP64 by the C restatement, on 10 seeded
  random directions;
* the checkpoint interval does not change the gradient (bit-identical);
* several windowed shots in one plan equal standalone runs on the cropped
  models (bit-identical seismograms) and the FP64 stack equals the sum of the
  per-shot gradients.
"""
import numpy as np
import pytest
import torch

from oracle import c_oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _smooth(a, k=3):
    from taichirtm_b200.synthetic import gaussian_smooth
    return gaussian_smooth(a, k)


def _problem(nx=72, nz=56, nt=320, fw=10, seed=7):
    rng = np.random.default_rng(seed)
    vp = 2200.0 + 400.0 * _smooth(rng.standard_normal((nx, nz)), 4) / 0.2
    vp = np.clip(vp, 1800.0, 2800.0)
    vs = vp / 1.8
    rho = 310.0 * vp ** 0.25
    t = np.arange(nt) / 2000.0
    a = (np.pi * 40.0 * (t - 0.025)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.array([[nx // 2, 3], [nx // 4, 6]], np.int32)
    wav = np.zeros((3, 2, nt), np.float32)
    wav[0, 0], wav[2, 0], wav[2, 1] = 0.3 * w, w, 0.6 * w
    rec = np.stack([np.arange(fw, nx - fw, 3), np.full(len(range(fw, nx - fw, 3)), 2)], 1).astype(np.int32)
    return dict(nx=nx, nz=nz, nt=nt, fw=fw, dx=5.0, dz=5.0, fs=2000.0, vp=vp, vs=vs, rho=rho, src=src,
                rec=rec, wav=wav)


def _fwi(P, ckpt=None, shots=None):
    from taichirtm_b200.fwi import FWIProblem
    from taichirtm_b200.plan import ShotGeometry
    shots = shots or [ShotGeometry(0, P["nx"], P["src"], P["rec"])]
    return FWIProblem(P["nx"], P["nz"], P["dx"], P["dz"], P["fs"], P["nt"], P["fw"], shots, P["wav"],
                      ckpt_every=ckpt)


def _lame(vp, vs, rho):
    mu = rho * vs ** 2
    return rho * vp ** 2 - 2 * mu, mu, rho


def test_dot_product_wavelet_adjoint():
    P = _problem()
    prob = _fwi(P, ckpt=17)
    lam, mu, rho = (torch.as_tensor(x, dtype=torch.float32) for x in _lame(P["vp"], P["vs"], P["rho"]))
    rng = np.random.default_rng(3)
    w = rng.standard_normal(P["wav"].shape).astype(np.float32)
    w[1] = 0
    prob.wavelets = torch.as_tensor(w).cuda()
    d, ck, flags = prob.forward(lam, mu, rho)
    g = rng.standard_normal(tuple(d.shape)).astype(np.float32)
    g[1] = 0
    _, gw = prob.adjoint(torch.as_tensor(g), ck, want_wavelet_grad=True)
    lhs = float((d.double().cpu().numpy()[[0, 2]] * g[[0, 2]].astype(np.float64)).sum())
    rhs = float((w[[0, 2]].astype(np.float64) * gw.double().cpu().numpy()[[0, 2]]).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)
    prob.close()


def _J_fp64(P, vp, vs, rho, obs):
    lam, mu, rho_ = _lame(vp, vs, rho)
    out = c_oracle.forward(mu, lam, rho_, dx=P["dx"], dz=P["dz"], nt=P["nt"], fs=P["fs"], fw=P["fw"],
                           src=P["src"], wu=P["wav"][0], wv=P["wav"][1], ww=P["wav"][2], rec=P["rec"],
                           dtype=np.float64, modes=1, check_interval=0)
    r = out["seis"][[0, 2]] - obs[[0, 2]]
    return 0.5 * float((r * r).sum())


def test_dot_product_model_parameters_fp64():
    """The adjoint as a linear operator in model space: for a random data-space
    cotangent g (all three components) and seeded smooth model directions dm,
    <J dm, g> with J dm the centred FP64 difference of the C restatement's
    seismograms equals <dm, J^T g> from the GPU adjoint (through the autograd
    path, w.r.t. vp, vs, rho), to 1e-4 relative."""
    from taichirtm_b200.fwi import seismograms
    P = _problem()
    rng = np.random.default_rng(211)
    prob = _fwi(P, ckpt=19)
    m = [torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in (P["vp"], P["vs"], P["rho"])]
    d = seismograms(m[0], m[1], m[2], prob)
    g = rng.standard_normal(tuple(d.shape))
    g[1] = 0.0  # P-SV only: the SH component is not driven by (vp, vs, rho) through this problem's sources
    d.backward(torch.as_tensor(g, dtype=d.dtype, device=d.device))
    jtg = [x.grad.cpu().numpy() for x in m]
    prob.close()

    def seis64(vp, vs, rho):
        lam, mu, rho_ = _lame(vp, vs, rho)
        return c_oracle.forward(mu, lam, rho_, dx=P["dx"], dz=P["dz"], nt=P["nt"], fs=P["fs"], fw=P["fw"],
                                src=P["src"], wu=P["wav"][0], wv=P["wav"][1], ww=P["wav"][2], rec=P["rec"],
                                dtype=np.float64, modes=1, check_interval=0)["seis"]

    errs = []
    for _ in range(3):
        dm = [_smooth(rng.standard_normal(P["vp"].shape), 2) for _ in range(3)]
        dm = [s * x / np.abs(x).max() for s, x in zip((P["vp"].mean(), P["vs"].mean(), P["rho"].mean()), dm)]
        eps = 1e-4
        dp = seis64(*(v + eps * x for v, x in zip((P["vp"], P["vs"], P["rho"]), dm)))
        dn = seis64(*(v - eps * x for v, x in zip((P["vp"], P["vs"], P["rho"]), dm)))
        jdm = (dp - dn) / (2 * eps)
        lhs = float((jdm[[0, 2]] * g[[0, 2]]).sum())
        rhs = sum(float((a * b).sum()) for a, b in zip(jtg, dm))
        errs.append(abs(lhs - rhs) / abs(lhs))
    print(f"model-space dot product: relative errors {['%.2e' % e for e in errs]}")
    assert max(errs) < 1e-4, errs


def test_gradient_vs_centred_finite_differences_fp64():
    """<grad J, dm> from the FP32 adjoint vs (J(m + e dm) - J(m - e dm)) / 2e
    with J evaluated by the FP64 C restatement of the same discrete forward."""
    from taichirtm_b200.fwi import l2_misfit
    P = _problem()
    rng = np.random.default_rng(104)
    vp_t = P["vp"] * (1 + 0.05 * _smooth(rng.standard_normal(P["vp"].shape), 3) / 0.2)
    lam_t, mu_t, rho_t = _lame(vp_t, vp_t / 1.8, 310.0 * vp_t ** 0.25)
    obs = c_oracle.forward(mu_t, lam_t, rho_t, dx=P["dx"], dz=P["dz"], nt=P["nt"], fs=P["fs"], fw=P["fw"],
                           src=P["src"], wu=P["wav"][0], wv=P["wav"][1], ww=P["wav"][2], rec=P["rec"],
                           dtype=np.float64, modes=1, check_interval=0)["seis"]
    prob = _fwi(P, ckpt=18)
    m = [torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in (P["vp"], P["vs"], P["rho"])]
    J = l2_misfit(m[0], m[1], m[2], prob, torch.as_tensor(obs.astype(np.float32)))
    J.backward()
    g = [x.grad.cpu().numpy() for x in m]
    errs = []
    for k in range(10):
        dm = [_smooth(rng.standard_normal(P["vp"].shape), 2) for _ in range(3)]
        dm = [d / np.abs(d).max() for d in dm]
        scale = [P["vp"].mean(), P["vs"].mean(), P["rho"].mean()]
        dm = [s * d for s, d in zip(scale, dm)]
        eps = 1e-4
        jp = _J_fp64(P, P["vp"] + eps * dm[0], P["vs"] + eps * dm[1], P["rho"] + eps * dm[2], obs)
        jm = _J_fp64(P, P["vp"] - eps * dm[0], P["vs"] - eps * dm[1], P["rho"] - eps * dm[2], obs)
        fd = (jp - jm) / (2 * eps)
        ad = sum(float((gi * di).sum()) for gi, di in zip(g, dm))
        errs.append(abs(ad - fd) / abs(fd))
    prob.close()
    assert max(errs) < 1e-4, errs


def test_checkpoint_interval_does_not_change_gradient():
    P = _problem(nt=200)
    lam, mu, rho = (torch.as_tensor(x, dtype=torch.float32) for x in _lame(P["vp"], P["vs"], P["rho"]))
    out = []
    for ck in (7, 200):
        prob = _fwi(P, ckpt=ck)
        d, c, _ = prob.forward(lam, mu, rho)
        grad, _ = prob.adjoint(d, c)
        out.append(grad.cpu().numpy())
        prob.close()
    assert np.array_equal(out[0], out[1])


def test_repeated_gradients_on_one_problem_are_identical():
    """The adjoint's scratch (recompute slots, gradient sums) stays with the
    plan from call to call and grows when a call needs more (here: the
    wavelet gradient): every call starts from cleared scratch, so repeated
    gradients are bit-identical."""
    P = _problem(nt=200)
    lam, mu, rho = (torch.as_tensor(x, dtype=torch.float32) for x in _lame(P["vp"], P["vs"], P["rho"]))
    prob = _fwi(P, ckpt=11)
    d, c, _ = prob.forward(lam, mu, rho)
    g1, _ = prob.adjoint(d, c)
    g2, gw = prob.adjoint(d, c, want_wavelet_grad=True)
    g3, _ = prob.adjoint(d, c)
    _, gw2 = prob.adjoint(d, c, want_wavelet_grad=True)
    assert np.abs(g1.cpu().numpy()).max() > 0
    assert np.array_equal(g1.cpu().numpy(), g2.cpu().numpy())
    assert np.array_equal(g1.cpu().numpy(), g3.cpu().numpy())
    assert np.array_equal(gw.cpu().numpy(), gw2.cpu().numpy())
    prob.close()


def test_two_steps_per_launch_adjoint_is_taken_and_equal():
    """With two steps per launch the segment recompute and the reverse sweep
    run in pairs (about half the launches of one step per launch, not a
    silent fallback), and the gradient is bit-identical."""
    P = _problem(nt=200)
    lam, mu, rho = _lame(P["vp"], P["vs"], P["rho"])
    from taichirtm_b200.fwi import FWIProblem
    from taichirtm_b200.plan import ShotGeometry
    out = {}
    for ts in (1, 2):
        prob = FWIProblem(P["nx"], P["nz"], P["dx"], P["dz"], P["fs"], P["nt"], P["fw"],
                          [ShotGeometry(0, P["nx"], P["src"], P["rec"])], P["wav"], ckpt_every=15,
                          tune=dict(vec=2, rows=8, warps=2, tsteps=ts))
        seis, ck, _ = prob.forward(lam, mu, rho)
        g, _ = prob.adjoint(seis * 0.3, ck)
        out[ts] = (g.cpu().numpy(), prob.plan.launch_count())
        prob.close()
    assert np.abs(out[1][0]).max() > 0
    assert np.array_equal(out[1][0], out[2][0])
    # one step per launch: 200 reversed steps plus the recompute and folds
    assert out[1][1] >= 200 + 180
    assert out[2][1] < 0.6 * out[1][1], (out[1][1], out[2][1])


def test_windowed_shots_equal_cropped_standalone_runs():
    from taichirtm_b200.plan import Plan, ShotGeometry
    rng = np.random.default_rng(9)
    nx, nz, nt, fw = 220, 60, 180, 12
    vp = 2000 + 600 * _smooth(rng.standard_normal((nx, nz)), 5) / 0.2
    vp = np.clip(vp, 1600, 2900)
    lam, mu, rho = _lame(vp, vp / 1.8, 310 * vp ** 0.25)
    lam, mu, rho = (x.astype(np.float32) for x in (lam, mu, rho))
    t = np.arange(nt) / 2000.0
    a = (np.pi * 40.0 * (t - 0.025)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    shots = []
    for x0, n, s in [(0, 90, 40), (50, 110, 60), (130, 90, 45)]:
        rec = np.stack([np.arange(fw, n - fw, 2), np.ones(len(range(fw, n - fw, 2)), int)], 1)
        shots.append(ShotGeometry(x0, n, [[s, 2]], rec))
    wav = np.zeros((3, len(shots), nt), np.float32)
    wav[2] = w
    wav[0] = 0.2 * w
    batch = Plan(nx, nz, 5.0, 5.0, nt, 2000.0, fw, 1, shots, tune=dict(vec=2, rows=16, warps=4))
    batch.set_model(mu, lam, rho)
    _, seis_b, _, _ = batch.forward(torch.as_tensor(wav), save=False)
    seis_b = seis_b.cpu().numpy()
    r0 = 0
    for k, s in enumerate(shots):
        one = Plan(s.nx, nz, 5.0, 5.0, nt, 2000.0, fw, 1, [ShotGeometry(0, s.nx, s.src, s.rec)])
        one.set_model(mu[s.x0:s.x0 + s.nx], lam[s.x0:s.x0 + s.nx], rho[s.x0:s.x0 + s.nx])
        _, seis1, _, _ = one.forward(torch.as_tensor(wav[:, k:k + 1]), save=False)
        nr = len(s.rec)
        assert np.array_equal(seis_b[:, r0:r0 + nr], seis1.cpu().numpy()), k
        r0 += nr
        one.close()
    batch.close()


def test_batched_gradient_is_sum_of_shot_gradients():
    from taichirtm_b200.fwi import FWIProblem
    from taichirtm_b200.plan import ShotGeometry
    P = _problem(nx=120, nz=50, nt=160)
    lam, mu, rho = (torch.as_tensor(x, dtype=torch.float32) for x in _lame(P["vp"], P["vs"], P["rho"]))
    shots = [ShotGeometry(0, 70, [[30, 3]], [[i, 2] for i in range(10, 60, 4)]),
             ShotGeometry(45, 75, [[40, 3]], [[i, 2] for i in range(10, 65, 5)])]
    wav = np.zeros((3, 2, P["nt"]), np.float32)
    wav[2] = P["wav"][2, 0]
    rng = np.random.default_rng(5)
    both = FWIProblem(P["nx"], P["nz"], 5.0, 5.0, 2000.0, P["nt"], P["fw"], shots, wav, ckpt_every=13)
    d, ck, _ = both.forward(lam, mu, rho)
    g = torch.as_tensor(rng.standard_normal(tuple(d.shape)).astype(np.float32))
    grad_both, _ = both.adjoint(g, ck)
    total = torch.zeros_like(grad_both)
    r0 = 0
    for k, s in enumerate(shots):
        one = FWIProblem(P["nx"], P["nz"], 5.0, 5.0, 2000.0, P["nt"], P["fw"], [s], wav[:, k:k + 1], ckpt_every=13)
        d1, ck1, _ = one.forward(lam, mu, rho)
        nr = len(s.rec)
        assert torch.equal(d1, d[:, r0:r0 + nr])
        gr, _ = one.adjoint(g[:, r0:r0 + nr].contiguous(), ck1)
        total += gr
        r0 += nr
        one.close()
    both.close()
    assert rel_l2(grad_both.cpu().numpy(), total.cpu().numpy()) < 1e-12


def _windowed_case(nt=200, seed=9):
    from taichirtm_b200.plan import ShotGeometry
    rng = np.random.default_rng(seed)
    nx, nz, fw = 220, 60, 12
    vp = np.clip(2000 + 600 * _smooth(rng.standard_normal((nx, nz)), 5) / 0.2, 1600, 2900)
    lam, mu, rho = (x.astype(np.float32) for x in _lame(vp, vp / 1.8, 310 * vp ** 0.25))
    t = np.arange(nt) / 2000.0
    a = (np.pi * 40.0 * (t - 0.025)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    shots = []
    for x0, n, s in [(0, 90, 40), (50, 110, 60), (130, 90, 45)]:
        rec = np.stack([np.arange(fw, n - fw, 2), np.ones(len(range(fw, n - fw, 2)), int)], 1)
        shots.append(ShotGeometry(x0, n, [[s, 2]], rec))
    wav = np.zeros((3, len(shots), nt), np.float32)
    wav[2] = w
    wav[0] = 0.2 * w
    return dict(nx=nx, nz=nz, nt=nt, fw=fw, lam=lam, mu=mu, rho=rho, shots=shots, wav=wav)


def test_checkpointed_rtm_equals_snapshot_rtm_and_compressed_error():
    """FP32 checkpoints + recompute give the snapshot path's image bit for bit;
    the block-scaled 16-bit checkpoints stay close (errors printed), the
    int16 block-floating-point format closest."""
    from taichirtm_b200.batch import BatchedRTM
    C = _windowed_case()
    kw = dict(tune=dict(vec=2, rows=16, warps=4), graphs=False)
    true = BatchedRTM(C["mu"], C["lam"], 1.02 * C["rho"], 5.0, 5.0, 2000.0, C["nt"], C["fw"], C["shots"], **kw)
    _, obs, _, _ = true.forward(C["wav"])
    true.close()
    rtm = BatchedRTM(C["mu"], C["lam"], C["rho"], 5.0, 5.0, 2000.0, C["nt"], C["fw"], C["shots"], **kw)
    ff, fb, ref = rtm.migrate(C["wav"], obs, isnap=4)
    ref = ref.cpu().numpy()
    for every in (13, 200):
        _, _, st = rtm.migrate(C["wav"], obs, isnap=4, checkpoint=dict(every=every, dtype="f32"))
        assert np.array_equal(st.cpu().numpy(), ref), every
    errs = {}
    for dt in ("f16", "bf16", "i16"):
        _, _, st = rtm.migrate(C["wav"], obs, isnap=4, checkpoint=dict(every=13, dtype=dt))
        errs[dt] = rel_l2(st.cpu().numpy()[[0, 2]], ref[[0, 2]])
    print("compressed-checkpoint image rel-L2:", errs)
    assert errs["f16"] < 5e-3 and errs["bf16"] < 5e-2 and errs["i16"] < 1e-4, errs
    assert errs["i16"] < 0.25 * errs["f16"], errs
    rtm.close()


def test_compressed_checkpoint_gradient_error():
    from taichirtm_b200.fwi import FWIProblem
    P = _problem(nt=240)
    lam, mu, rho = (torch.as_tensor(x, dtype=torch.float32) for x in _lame(P["vp"], P["vs"], P["rho"]))
    rng = np.random.default_rng(11)
    out = {}
    for dt in ("f32", "f16", "bf16", "i16"):
        prob = _fwi(P, ckpt=16)
        prob = FWIProblem(P["nx"], P["nz"], P["dx"], P["dz"], P["fs"], P["nt"], P["fw"],
                          prob.plan.shots, P["wav"], ckpt_every=16, ckpt_dtype=dt)
        d, ck, _ = prob.forward(lam, mu, rho)
        g = torch.as_tensor(np.random.default_rng(11).standard_normal(tuple(d.shape)).astype(np.float32))
        grad, _ = prob.adjoint(g, ck)
        out[dt] = grad.cpu().numpy()
        prob.close()
    e16 = rel_l2(out["f16"], out["f32"])
    eb16 = rel_l2(out["bf16"], out["f32"])
    ei16 = rel_l2(out["i16"], out["f32"])
    print("compressed-checkpoint gradient rel-L2: f16 %.2e bf16 %.2e i16 %.2e" % (e16, eb16, ei16))
    assert e16 < 1e-2 and eb16 < 1e-1 and ei16 < 1e-4
    assert ei16 < 0.25 * e16


@pytest.mark.parametrize("dtype", ["f16", "i16"])
def test_compressed_checkpoints_independent_of_launch_shape(dtype):
    """The 16-bit checkpoints are scaled per 60-column block whatever the
    warp strip (60 columns at vec 2, 120 at vec 4), and written by the step
    launch that produces the state (one or two steps per launch): the
    gradient is bit-identical across these launch shapes."""
    from taichirtm_b200.fwi import FWIProblem
    from taichirtm_b200.plan import ShotGeometry
    P = _problem(nt=150)
    lam, mu, rho = _lame(P["vp"], P["vs"], P["rho"])
    grads = []
    for tune in (dict(vec=2, rows=8, warps=2, tsteps=1), dict(vec=2, rows=6, warps=2, tsteps=2, prefetch=3),
                 dict(vec=4, rows=5, warps=1, prefetch=1), dict(vec=4, rows=7, warps=2, tsteps=2)):
        prob = FWIProblem(P["nx"], P["nz"], P["dx"], P["dz"], P["fs"], P["nt"], P["fw"],
                          [ShotGeometry(0, P["nx"], P["src"], P["rec"])], P["wav"], ckpt_every=12, tune=tune,
                          ckpt_dtype=dtype)
        seis, ck, _ = prob.forward(lam, mu, rho)
        g, _ = prob.adjoint(seis * 0.3, ck)
        grads.append(g.cpu().numpy())
        prob.close()
    assert np.abs(grads[0]).max() > 0
    for g in grads[1:]:
        assert np.array_equal(grads[0], g)


def test_gradient_independent_of_launch_shape_and_autotuned():
    """The adjoint's per-cell arithmetic and its 64-step fold do not depend on
    the launch shape: FWIProblem(tune="auto") (timed on short gradients) and
    fixed shapes give bit-identical gradients.  With two steps per launch the
    forward recompute of each segment runs in pairs that store both states
    (an odd count ends with a single step: segments of 14 and 4 steps)."""
    P = _problem(nt=200)
    lam, mu, rho = _lame(P["vp"], P["vs"], P["rho"])
    grads = []
    for tune in ("auto", dict(vec=2, rows=8, warps=2, tsteps=2), dict(vec=4, rows=5, warps=1),
                 dict(vec=1, rows=3, warps=4), dict(vec=2, rows=8, warps=2, tsteps=2, prefetch=3),
                 dict(vec=4, rows=6, warps=3, prefetch=3), dict(vec=4, rows=7, warps=2, tsteps=2),
                 dict(vec=4, rows=6, warps=3, tsteps=2, prefetch=3), dict(vec=2, rows=8, warps=1, tsteps=2),
                 dict(vec=2, rows=5, warps=1, tsteps=2, prefetch=4), dict(vec=2, rows=7, warps=1)):
        from taichirtm_b200.fwi import FWIProblem
        from taichirtm_b200.plan import ShotGeometry
        prob = FWIProblem(P["nx"], P["nz"], P["dx"], P["dz"], P["fs"], P["nt"], P["fw"],
                          [ShotGeometry(0, P["nx"], P["src"], P["rec"])], P["wav"], ckpt_every=14, tune=tune)
        seis, ck, _ = prob.forward(lam, mu, rho)
        g, _ = prob.adjoint(seis * 0.3, ck)
        grads.append(g.cpu().numpy())
        prob.close()
    assert np.abs(grads[0]).max() > 0
    for g in grads[1:]:
        assert np.array_equal(grads[0], g)
