"""Error of every workload configuration's outputs against an FP64 run of the
reference algorithm (the C restatement in double), at the configuration's own
grid:

* 1001 x 501 SH RTM at full length (nt 4000, isnap 7): seismograms
  rel-L2 <= 1e-5, image rel-L2 <= 1e-4;
* the 4001 x 1601 model with two windowed shots and checkpointed RTM plus
  FWI gradient over 25 checkpoint segments: the image with 16-bit
  block-floating-point (int16) checkpoints <= 1e-4, and the gradient's
  directional derivatives on 3 seeded directions within 1e-4 of centred
  finite differences of the FP64 forward; FP16 and FP32 checkpoints are
  measured beside it;
* the 1201 x 401 FWI gradient at full length (nt 3000, sqrt(nt) FP32
  checkpoints, two of the eight shots) against centred FP64 finite
  differences on 3 seeded directions: within 1e-4.

The directional-derivative checks are the FP64 statement for the gradient:
the reference has no gradient to compare with, and the FP64 restatement has
no adjoint, so ``<grad J, dm>`` is compared with ``(J(m + e dm) - J(m - e dm))
/ 2e`` where J is evaluated by the FP64 forward.
"""
import math

import numpy as np
import pytest
import torch

from oracle import c_oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
IMG_TOL = 1e-4
GRAD_TOL = 1e-4


def _lame64(vp, vs, rho):
    vp, vs, rho = (np.asarray(x, np.float64) for x in (vp, vs, rho))
    mu = rho * vs ** 2
    return mu, rho * vp ** 2 - 2 * mu, rho


def test_config2_sh_rtm_full_length_vs_fp64_oracle():
    """1001 x 501 SH: observed data on the true model, forward with
    snapshots every 7 steps and backward with imaging on the migration model,
    all 4000 steps, through the reference-shaped classes."""
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    from taichirtm_b200 import synthetic as S
    s = S.config2()
    sh = s.shots[0]
    mu, lam, rho = s.material()
    mum, lamm, rhom = s.material(migration=True)
    kw = dict(dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, fw=s.fw, dtype=np.float64, modes=2)
    wv = dict(wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2])
    ref_obs = c_oracle.forward(mu, lam, rho, src=sh.src, rec=sh.rec, **wv, **kw)
    ref_fw = c_oracle.forward(mum, lamm, rhom, src=sh.src, rec=sh.rec, save=True, isnap=7, snap_comps=(1,),
                              **wv, **kw)
    ref_img = c_oracle.backward(mum, lamm, rhom, rec=sh.rec, obs=ref_obs["seis"], snaps=ref_fw["snaps"],
                                isnaps=ref_fw["isnaps"], num_snaps=ref_fw["num_snaps"], isnap=7, snap_comps=(1,),
                                **kw)["img"]
    del ref_fw
    c = dict(nx=s.nx, nz=s.nz, dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, absorbing_frame=s.fw,
             src_loc_field=sh.src, recv_loc_field=sh.rec, num_sources=1, num_receivers=len(sh.rec))
    wav = dict(wavelet_u_field=sh.wavelets[0], wavelet_v_field=sh.wavelets[1], wavelet_w_field=sh.wavelets[2])
    fo = ForwardModeling(isnap=7, mu_field=mu, lam_field=lam, rho_field=rho, **c, **wav)
    assert fo.modes == 2 and fo.run() == 0
    obs = np.stack(fo.get_seismogram())
    e_seis = rel_l2(obs[1], ref_obs["seis"][1])
    fo.cleanup()
    fm = ForwardModeling(isnap=7, mu_field=mum, lam_field=lamm, rho_field=rhom, **c, **wav)
    assert fm.run(save=True) == 0
    bw = BackwardModeling(obsdata_u_field=obs[0], obsdata_v_field=obs[1], obsdata_w_field=obs[2],
                          mu_field=mum, lam_field=lamm, rho_field=rhom, **c)
    assert bw.run_calc(fm.u_save_field, fm.v_save_field, fm.w_save_field, fm.isnaps_field, fm.num_snaps, 7) == 0
    img = np.stack(bw.get_results())
    e_img = rel_l2(img[1], ref_img[1])
    print(f"config 2 SH full length vs FP64: seismogram {e_seis:.2e}, image {e_img:.2e}")
    assert e_seis <= SEIS_TOL, e_seis
    assert e_img <= IMG_TOL, e_img
    fm.cleanup()
    bw.cleanup()


def _fp64_seis(sv, shots, vp, vs, rho):
    """FP64 seismograms (3, nrec_total, nt) of the shots on their windows."""
    mu, lam, rh = _lame64(vp, vs, rho)
    out = []
    for s in shots:
        crop = [np.ascontiguousarray(x[s.x0:s.x0 + s.nx]) for x in (mu, lam, rh)]
        f = c_oracle.forward(*crop, dx=sv.dx, dz=sv.dz, nt=sv.nt, fs=sv.fs, fw=sv.fw, src=s.src, wu=s.wavelets[0],
                             wv=s.wavelets[1], ww=s.wavelets[2], rec=s.rec, dtype=np.float64, modes=1,
                             check_interval=0)
        out.append(f["seis"])
    return np.concatenate(out, axis=1)


def _directions(shape, scale, rng, n):
    from taichirtm_b200.synthetic import gaussian_smooth
    dirs = []
    for _ in range(n):
        dm = [gaussian_smooth(rng.standard_normal(shape), 6.0) for _ in range(3)]
        dirs.append([s * d / np.abs(d).max() for s, d in zip(scale, dm)])
    return dirs


def _fd_check(sv, shots, m0, obs, grads, dirs, eps=1e-4):
    """Relative errors of <g, dm> against centred FP64 differences of J."""
    def J(m):
        r = _fp64_seis(sv, shots, *m)[[0, 2]] - obs[[0, 2]]
        return 0.5 * float((r * r).sum())
    errs = {k: [] for k in grads}
    for dm in dirs:
        jp = J([x + eps * d for x, d in zip(m0, dm)])
        jm = J([x - eps * d for x, d in zip(m0, dm)])
        fd = (jp - jm) / (2 * eps)
        for k, g in grads.items():
            ad = sum(float((gi * di).sum()) for gi, di in zip(g, dm))
            errs[k].append(abs(ad - fd) / abs(fd))
    return errs


def test_large_model_checkpointed_rtm_and_gradient_vs_fp64():
    """Two windowed shots of the 4001 x 1601 model, nt 600 (checkpoints every
    24 steps: 25 segments).  Image of checkpointed RTM (isnap 16) and FWI
    gradient with FP32, FP16 and int16 block-floating-point checkpoints
    against FP64: int16 and FP32 within 1e-4; FP16 reported."""
    from taichirtm_b200 import synthetic as S
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.fwi import FWIProblem, l2_misfit
    from taichirtm_b200.plan import ShotGeometry
    sv = S.config5(nt=600)
    sub = sv.shots[:2]
    geo = [ShotGeometry(s.x0, s.nx, s.src, s.rec) for s in sub]
    K = round(math.sqrt(sv.nt))
    assert (sv.nt + K - 1) // K >= 9
    m0 = [sv.vp_mig, sv.vs_mig, sv.rho_mig]
    mu, lam, rho = _lame64(*m0)
    # FP64: forward with snapshots and backward with imaging per shot, the
    # observed data being half the migration model's own FP64 seismograms
    img64 = np.zeros((3, sv.nx, sv.nz))
    obs_parts, seis64 = [], []
    for s in sub:
        crop = [np.ascontiguousarray(x[s.x0:s.x0 + s.nx]) for x in (mu, lam, rho)]
        kw = dict(dx=sv.dx, dz=sv.dz, nt=sv.nt, fs=sv.fs, fw=sv.fw, dtype=np.float64, modes=1)
        f = c_oracle.forward(*crop, src=s.src, wu=s.wavelets[0], wv=s.wavelets[1], ww=s.wavelets[2], rec=s.rec,
                             save=True, isnap=16, snap_comps=(0, 2), **kw)
        o = (0.5 * f["seis"]).astype(np.float32)
        b = c_oracle.backward(*crop, rec=s.rec, obs=o, snaps=f["snaps"], isnaps=f["isnaps"],
                              num_snaps=f["num_snaps"], isnap=16, snap_comps=(0, 2), **kw)
        img64[:, s.x0:s.x0 + s.nx] += b["img"]
        obs_parts.append(o)
        seis64.append(f["seis"])
        del f
    obs = np.concatenate(obs_parts, axis=1)
    wav = np.concatenate([s.wavelets for s in sub], axis=1)
    mu32, lam32, rho32 = sv.material(migration=True)
    tune = dict(vec=2, rows=32, warps=1, tsteps=2, prefetch=3)
    rtm = BatchedRTM(mu32, lam32, rho32, sv.dx, sv.dz, sv.fs, sv.nt, sv.fw, geo, tune=tune, graphs=False)
    _, seis, _, _ = rtm.forward(wav)
    seis_err = rel_l2(seis.cpu().numpy()[[0, 2]], np.concatenate(seis64, axis=1)[[0, 2]])
    img_err = {}
    for dt in ("f32", "f16", "i16"):
        ff, fb, st = rtm.migrate(wav, obs, isnap=16, checkpoint=dict(every=K, dtype=dt))
        assert int(ff.max()) == 0 and int(fb.max()) == 0
        img_err[dt] = rel_l2(st.cpu().numpy()[[0, 2]], img64[[0, 2]])
    rtm.close()
    # gradient of 0.5 ||d - obs||^2 at m0 for each checkpoint storage
    grads = {}
    for dt in ("f32", "f16", "i16"):
        prob = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, sv.nt, sv.fw, geo, wav, ckpt_every=K, tune=tune,
                          ckpt_dtype=dt)
        m = [torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in m0]
        l2_misfit(m[0], m[1], m[2], prob, torch.as_tensor(obs)).backward()
        grads[dt] = [x.grad.cpu().numpy() for x in m]
        prob.close()
    rng = np.random.default_rng(105)
    dirs = _directions(sv.vp.shape, [np.mean(x) for x in m0], rng, 3)
    grad_err = _fd_check(sv, sub, m0, obs.astype(np.float64), grads, dirs)
    flat = {k: np.concatenate([g.ravel() for g in v]) for k, v in grads.items()}
    print(f"large model vs FP64: seismograms {seis_err:.2e}, image", {k: f"{v:.2e}" for k, v in img_err.items()},
          "gradient directional", {k: f"{max(v):.2e}" for k, v in grad_err.items()},
          "gradient rel-L2 vs FP32 checkpoints: f16 %.2e i16 %.2e" % (rel_l2(flat["f16"], flat["f32"]),
                                                                       rel_l2(flat["i16"], flat["f32"])))
    assert seis_err <= SEIS_TOL, seis_err
    assert img_err["f32"] <= IMG_TOL and img_err["i16"] <= IMG_TOL, img_err
    assert max(grad_err["f32"]) <= GRAD_TOL and max(grad_err["i16"]) <= GRAD_TOL, grad_err
    assert img_err["f16"] <= 1e-3, img_err  # reported; FP16 keeps 11 bits per value


def test_config4_gradient_full_size_vs_fp64_finite_differences():
    """The 1201 x 401 FWI gradient at nt 3000 with sqrt(nt) FP32 checkpoints
    (two of the eight shots: the gradient is a sum over shots), observed data
    from the true model, against centred FP64 differences of J on 3 seeded
    directions and along the gradient itself.

    Two gradients are compared.  The adjoint driven by the FP64 residual
    d64(m0) - d_obs (rounded once to FP32) isolates the discrete adjoint and
    its FP32 arithmetic: within 1e-4 in every direction.  The end-to-end
    gradient of l2_misfit uses the FP32 forward's own residual; the smoothed
    starting model leaves a residual much smaller than the data, so the FP32
    seismogram error (relative to the data) grows by ||d|| / ||r|| relative
    to the residual, and the gradient is linear in the residual.  Its errors
    are held to 1e-4 along the gradient and, in the random directions, to
    that amplified FP32 floor (both printed)."""
    from taichirtm_b200 import synthetic as S
    from taichirtm_b200.fwi import FWIProblem, chain_to_lame_rho, l2_misfit
    from taichirtm_b200.plan import ShotGeometry
    sv = S.config4()
    sub = [sv.shots[1], sv.shots[5]]
    geo = [ShotGeometry(s.x0, s.nx, s.src, s.rec) for s in sub]
    wav = np.concatenate([s.wavelets for s in sub], axis=1)
    obs = _fp64_seis(sv, sub, sv.vp, sv.vs, sv.rho).astype(np.float32)
    m0 = [sv.vp_mig, sv.vs_mig, sv.rho_mig]
    d64 = _fp64_seis(sv, sub, *m0)
    K = round(math.sqrt(sv.nt))
    prob = FWIProblem(sv.nx, sv.nz, sv.dx, sv.dz, sv.fs, sv.nt, sv.fw, geo, wav, ckpt_every=K,
                      tune=dict(vec=2, rows=16, warps=2, tsteps=2))
    m = [torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in m0]
    l2_misfit(m[0], m[1], m[2], prob, torch.as_tensor(obs)).backward()
    g_e2e = [x.grad.cpu().numpy() for x in m]
    # the adjoint driven by the FP64 residual, mapped to (vp, vs, rho) like the
    # autograd function does (fwi.py: chain_to_lame_rho, then mu = rho vs^2,
    # lam = rho vp^2 - 2 mu)
    mu0, lam0, rho0 = (torch.as_tensor(x.astype(np.float32)) for x in _lame64(*m0))
    d, ck, _ = prob.forward(lam0, mu0, rho0)
    seis_err = rel_l2(d.cpu().numpy()[[0, 2]], d64[[0, 2]])
    r64 = d64 - obs.astype(np.float64)
    r64[1] = 0.0
    gcoef, _ = prob.adjoint(torch.as_tensor(r64.astype(np.float32)), ck)
    prob.close()
    vp, vs, rho = (torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in m0)
    mu_t = rho * vs * vs
    lam_t = rho * vp * vp - 2.0 * mu_t
    g_lam, g_mu, g_rho = chain_to_lame_rho(gcoef, mu_t.detach(), rho.detach())
    torch.autograd.backward([lam_t, mu_t, rho], [g_lam, g_mu, g_rho])
    g_adj = [vp.grad.cpu().numpy(), vs.grad.cpu().numpy(), rho.grad.cpu().numpy()]
    kappa = float(np.linalg.norm(d64[[0, 2]]) / np.linalg.norm(r64[[0, 2]]))
    rng = np.random.default_rng(104)
    dirs = _directions(sv.vp.shape, [np.mean(x) for x in m0], rng, 3)
    dirs.append([gi / np.abs(gi).max() * np.mean(pi) for gi, pi in zip(g_adj, m0)])  # along the gradient
    errs = _fd_check(sv, sub, m0, obs.astype(np.float64), {"adjoint": g_adj, "end_to_end": g_e2e}, dirs)
    floor = seis_err * kappa
    print(f"config 4 vs FP64: seismograms {seis_err:.2e}; ||d||/||r|| {kappa:.1f} (FP32 floor relative to the "
          f"residual {floor:.1e}); directional errors (3 random, along the gradient): adjoint "
          f"{[f'{e:.2e}' for e in errs['adjoint']]}, end to end {[f'{e:.2e}' for e in errs['end_to_end']]}")
    assert seis_err <= SEIS_TOL, seis_err
    assert max(errs["adjoint"]) <= GRAD_TOL, errs
    assert errs["end_to_end"][-1] <= GRAD_TOL, errs
    assert max(errs["end_to_end"]) <= max(GRAD_TOL, 2.0 * floor), (errs, floor)
