"""GPU parity: the fused sm_100a kernels (through the reference-facing Python API
and the C ABI) against the golden vectors recorded from the reference source
and against the FP64 oracle.

Tolerances (against FP64 runs of the reference algorithm):
  seismograms  relative L2 <= 1e-5
  images       relative L2 <= 1e-4
"""
import numpy as np
import pytest
import torch

from oracle import c_oracle
from tests.conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
IMG_TOL = 1e-4


def _fields(g, which):
    return dict(mu_field=g["mu_" + which], lam_field=g["lam_" + which], rho_field=g["rho_" + which])


def _common(g):
    sm = g["surface"] if g["surface"].size else None
    return dict(nx=int(g["nx"]), nz=int(g["nz"]), dx=float(g["dx"]), dz=float(g["dz"]), nt=int(g["nt"]),
                fs=float(g["fs"]), absorbing_frame=int(g["fw"]), src_loc_field=g["src"],
                recv_loc_field=g["rec"], surface_matrix_field=sm, num_sources=len(g["src"]),
                num_receivers=len(g["rec"]))


@pytest.mark.parametrize("name", ["fwbw_basic", "fwbw_topo", "fwbw_narrow"])
def test_golden_forward_backward(name):
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    g = load_golden(name)
    c = _common(g)
    wav = dict(wavelet_u_field=g["wu"], wavelet_v_field=g["wv"], wavelet_w_field=g["ww"])
    fo = ForwardModeling(isnap=int(g["isnap"]), **c, **wav, **_fields(g, "t"))
    assert fo.run(save=False) == 0
    obs = np.stack(fo.get_seismogram())
    assert rel_l2(obs, g["obs"]) <= SEIS_TOL, rel_l2(obs, g["obs"])
    fs_ = ForwardModeling(isnap=int(g["isnap"]), **c, **wav, **_fields(g, "s"))
    assert fs_.run(save=True) == 0
    syn = np.stack(fs_.get_seismogram())
    assert rel_l2(syn, g["syn"]) <= SEIS_TOL
    snaps = np.stack([fs_.u_save_field.to_numpy(), fs_.v_save_field.to_numpy(), fs_.w_save_field.to_numpy()])
    assert snaps.shape == g["snaps"].shape
    assert rel_l2(snaps, g["snaps"]) <= SEIS_TOL
    assert np.array_equal(fs_.isnaps_field.to_numpy(), g["isnaps"])
    bw = BackwardModeling(obsdata_u_field=g["obs"][0], obsdata_v_field=g["obs"][1],
                          obsdata_w_field=g["obs"][2], **c, **_fields(g, "s"))
    assert bw.run_calc(fs_.u_save_field, fs_.v_save_field, fs_.w_save_field, fs_.isnaps_field,
                       fs_.num_snaps, int(g["isnap"])) == 0
    img = np.stack(bw.get_results())
    for k in range(3):
        if np.abs(g["img"][k]).max() > 0:
            assert rel_l2(img[k], g["img"][k]) <= IMG_TOL, (k, rel_l2(img[k], g["img"][k]))
        else:
            assert np.abs(img[k]).max() == 0
    # snapshots given as plain NumPy (nx, nz, nsnap) arrays give the same image
    bw2 = BackwardModeling(obsdata_u_field=g["obs"][0], obsdata_v_field=g["obs"][1],
                           obsdata_w_field=g["obs"][2], **c, **_fields(g, "s"))
    assert bw2.run_calc(g["snaps"][0], g["snaps"][1], g["snaps"][2], g["isnaps"], int(g["num_snaps"]),
                        int(g["isnap"])) == 0
    assert rel_l2(np.stack(bw2.get_results()), g["img"]) <= IMG_TOL
    for o in (fo, fs_, bw, bw2):
        o.cleanup()


def test_edge_source_reports_code_3():
    """Source on an edge cell: inv_rho_u = 1/0 -> non-finite; the first check
    (it = 0) returns 3 like the reference (fm:304-307, 437-443, 471-472)."""
    from taichirtm_b200 import ForwardModeling
    g = load_golden("fwbw_edge_source")
    fm = ForwardModeling(isnap=2, wavelet_u_field=g["wu"], wavelet_v_field=g["wv"],
                         wavelet_w_field=g["ww"], **_common(g), **_fields(g, "s"))
    assert fm.run(save=True) == 3
    # with the check off the run continues and the NaN/inf pattern matches
    assert fm.run(save=False, stability_check_interval=10 ** 9) == 3  # it = 0 is still checked
    fm.cleanup()


def _c1_inputs(nt):
    from taichirtm_b200 import synthetic as S
    s = S.config1(nt=nt)
    return s, s.shots[0]


def test_config1_psv_rtm_vs_fp64_oracle():
    """301 x 151 P-SV RTM at full length (nt = 2000, isnap = 1) vs the FP64 C
    restatement: seismogram rel-L2 <= 1e-5, image rel-L2 <= 1e-4."""
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    s, sh = _c1_inputs(2000)
    mu, lam, rho = s.material()
    mum, lamm, rhom = s.material(migration=True)
    kw = dict(dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, fw=s.fw)
    ref_obs = c_oracle.forward(mu, lam, rho, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1],
                               ww=sh.wavelets[2], rec=sh.rec, dtype=np.float64, modes=1, **kw)
    ref_fw = c_oracle.forward(mum, lamm, rhom, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1],
                              ww=sh.wavelets[2], rec=sh.rec, dtype=np.float64, modes=1, save=True,
                              isnap=1, **kw)
    ref_img = c_oracle.backward(mum, lamm, rhom, rec=sh.rec, obs=ref_obs["seis"], snaps=ref_fw["snaps"],
                                isnaps=ref_fw["isnaps"], num_snaps=ref_fw["num_snaps"], isnap=1,
                                dtype=np.float64, modes=1, **kw)["img"]
    c = dict(nx=s.nx, nz=s.nz, dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, absorbing_frame=s.fw,
             src_loc_field=sh.src, recv_loc_field=sh.rec, num_sources=1, num_receivers=len(sh.rec))
    wav = dict(wavelet_u_field=sh.wavelets[0], wavelet_v_field=sh.wavelets[1], wavelet_w_field=sh.wavelets[2])
    fo = ForwardModeling(isnap=1, mu_field=mu, lam_field=lam, rho_field=rho, **c, **wav)
    assert fo.modes == 1
    assert fo.run() == 0
    obs = np.stack(fo.get_seismogram())
    e_seis = rel_l2(obs[[0, 2]], ref_obs["seis"][[0, 2]])
    assert e_seis <= SEIS_TOL, e_seis
    fm = ForwardModeling(isnap=1, mu_field=mum, lam_field=lamm, rho_field=rhom, **c, **wav)
    assert fm.run(save=True) == 0
    bw = BackwardModeling(obsdata_u_field=obs[0], obsdata_v_field=obs[1], obsdata_w_field=obs[2],
                          mu_field=mum, lam_field=lamm, rho_field=rhom, **c)
    assert bw.run_calc(fm.u_save_field, fm.v_save_field, fm.w_save_field, fm.isnaps_field, fm.num_snaps, 1) == 0
    img = np.stack(bw.get_results())
    e_img = rel_l2(img[[0, 2]], ref_img[[0, 2]])
    print(f"config 1 P-SV RTM vs FP64: seismograms {e_seis:.2e}, image {e_img:.2e}")
    assert e_img <= IMG_TOL, e_img
    assert np.abs(img[1]).max() == 0


def test_config2_sh_vs_fp64_oracle_short():
    """1001 x 501 SH propagation (nt shortened to 600) vs the FP64 oracle."""
    from taichirtm_b200 import ForwardModeling
    from taichirtm_b200 import synthetic as S
    s = S.config2(nt=600)
    sh = s.shots[0]
    mu, lam, rho = s.material()
    ref = c_oracle.forward(mu, lam, rho, dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, fw=s.fw, src=sh.src,
                           wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2], rec=sh.rec,
                           dtype=np.float64, modes=2)
    fo = ForwardModeling(nx=s.nx, nz=s.nz, dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, absorbing_frame=s.fw,
                         isnap=7, src_loc_field=sh.src, recv_loc_field=sh.rec, num_sources=1,
                         num_receivers=len(sh.rec), wavelet_u_field=sh.wavelets[0],
                         wavelet_v_field=sh.wavelets[1], wavelet_w_field=sh.wavelets[2],
                         mu_field=mu, lam_field=lam, rho_field=rho)
    assert fo.modes == 2
    assert fo.run() == 0
    e = rel_l2(np.stack(fo.get_seismogram())[1], ref["seis"][1])
    assert e <= SEIS_TOL, e


@pytest.mark.parametrize("tune", [dict(vec=1, rows=7, warps=2, prefetch=0), dict(vec=2, rows=16, warps=4, prefetch=1), dict(vec=2, rows=9, warps=3, prefetch=3), dict(vec=4, rows=16, warps=2, prefetch=3), dict(vec=1, rows=3, warps=2, prefetch=3),
                                  dict(vec=4, rows=64, warps=8, prefetch=0), dict(vec=2, rows=5, warps=1, prefetch=1)])
def test_launch_shapes_agree(tune):
    """Every launch shape gives the same seismograms and images (bit-exact:
    each cell's arithmetic does not depend on the decomposition)."""
    from taichirtm_b200.plan import Plan, ShotGeometry
    g = load_golden("fwbw_basic")
    nx, nz, nt = int(g["nx"]), int(g["nz"]), int(g["nt"])
    out = []
    for t in (None, tune):
        p = Plan(nx, nz, float(g["dx"]), float(g["dz"]), nt, float(g["fs"]), int(g["fw"]), 3,
                 [ShotGeometry(0, nx, g["src"], g["rec"])], tune=t)
        p.set_model(g["mu_s"], g["lam_s"], g["rho_s"])
        wav = torch.as_tensor(np.stack([g["wu"], g["wv"], g["ww"]]))
        f, seis, snaps, isn = p.forward(wav, save=True, isnap=3)
        f2, img, _ = p.backward(torch.as_tensor(g["obs"]).float(), snaps, isn, len(isn), 3)
        out.append((seis.cpu().numpy(), img.cpu().numpy()))
        p.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_cuda_graph_replay_matches_direct_launches():
    """tune.graphs = 1 captures each time loop once and replays it; results
    equal direct launches, on the capture call and on replays, and a changed
    snapshot schedule triggers a new capture."""
    from taichirtm_b200.plan import Plan, ShotGeometry
    g = load_golden("fwbw_basic")
    nx, nz, nt = int(g["nx"]), int(g["nz"]), int(g["nt"])
    wav = torch.as_tensor(np.stack([g["wu"], g["wv"], g["ww"]]))
    obs = torch.as_tensor(g["obs"]).float()
    res = {}
    for graphs in (0, 1):
        p = Plan(nx, nz, float(g["dx"]), float(g["dz"]), nt, float(g["fs"]), int(g["fw"]), 3,
                 [ShotGeometry(0, nx, g["src"], g["rec"])], tune=dict(graphs=graphs))
        p.set_model(g["mu_s"], g["lam_s"], g["rho_s"])
        out = []
        for isnap in (3, 3, 5):
            snaps = [p.snapshot_buffer(nt // isnap) for _ in range(3)]
            f, seis, snaps, isn = p.forward(wav, save=True, isnap=isnap, snaps=snaps)
            f2, img, _ = p.backward(obs, snaps, isn, len(isn), isnap)
            out.append((seis.cpu().numpy(), img.cpu().numpy()))
        res[graphs] = out
        p.close()
    for k in range(3):
        assert np.array_equal(res[0][k][0], res[1][k][0])
        assert np.array_equal(res[0][k][1], res[1][k][1])


@pytest.mark.parametrize("name", ["fwbw_basic", "fwbw_topo"])
def test_bit_exact_vs_fp32_restatement(name):
    """With FMA contraction off, each cell's FP32 arithmetic on the GPU is the
    reference's expression order; the NumPy FP32 restatement with the same
    one-time FP64 set-up and Kahan imaging gives identical bits."""
    from oracle import fd_oracle
    from taichirtm_b200.plan import Plan, ShotGeometry
    g = load_golden(name)
    sm = g["surface"] if g["surface"].size else None
    nx, nz, nt, isnap = int(g["nx"]), int(g["nz"]), int(g["nt"]), int(g["isnap"])
    kw = dict(dx=float(g["dx"]), dz=float(g["dz"]), nt=nt, fs=float(g["fs"]), fw=int(g["fw"]))
    ref = fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], src=g["src"], wu=g["wu"], wv=g["wv"],
                            ww=g["ww"], rec=g["rec"], isnap=isnap, surface=sm, save=True,
                            dtype=np.float32, setup_f64=True, **kw)
    bref = fd_oracle.backward(g["mu_s"], g["lam_s"], g["rho_s"], rec=g["rec"], ou=g["obs"][0],
                              ov=g["obs"][1], ow=g["obs"][2], snaps=ref["snaps"], isnaps=ref["isnaps"],
                              num_snaps=ref["num_snaps"], isnap=isnap, surface=sm, dtype=np.float32,
                              setup_f64=True, kahan=True, **kw)
    p = Plan(nx, nz, kw["dx"], kw["dz"], nt, kw["fs"], kw["fw"], 3, [ShotGeometry(0, nx, g["src"], g["rec"])])
    p.set_model(g["mu_s"], g["lam_s"], g["rho_s"], sm)
    f, seis, snaps, isn = p.forward(torch.as_tensor(np.stack([g["wu"], g["wv"], g["ww"]])), save=True,
                                    isnap=isnap)
    assert np.array_equal(seis.cpu().numpy(), ref["seis"])
    for c in range(3):
        assert np.array_equal(p.snapshot_view(snaps[c], len(isn)).cpu().numpy(), ref["snaps"][c])
    f2, img, _ = p.backward(torch.as_tensor(g["obs"]).float(), snaps, isn, len(isn), isnap)
    assert np.array_equal(img.cpu().numpy(), bref["img"])
    p.close()


@pytest.mark.parametrize("name", ["rtm_vfix", "rtm_vscan_topo"])
def test_reverse_time_migration_run_golden(name):
    """ReverseTimeMigration.run end to end (rtm.py:846-1029) vs the reference
    source run in FP64 on the same inputs."""
    from taichirtm_b200 import ReverseTimeMigration
    g = load_golden(name)
    r = ReverseTimeMigration()
    r.set_observed_data(g["obs"][0], g["obs"][1], g["obs"][2])
    r.set_source(g["src_w"][0], g["src_w"][1], g["src_w"][2], float(g["src_x"]))
    r.set_receivers(g["rec_x"]).set_frequency(float(g["fs"])).set_boundary(int(g["fw"]))
    r.set_velocity_range(float(g["vmin"]), float(g["vmax"]), int(g["vstep"]))
    r.set_poisson_ratio(float(g["poisson"]))
    if np.isfinite(g["v_fix"]):
        r.fix_velocity(float(g["v_fix"]))
    if g["heights"].size:
        r.set_topography(g["heights"])
    r.run()
    assert r.nx == int(g["nx"]) and r.nz == int(g["nz"])
    assert r.dx == pytest.approx(float(g["dx"]), rel=1e-12)
    assert r.CFL == pytest.approx(float(g["cfl"]))
    assert np.array_equal(np.asarray(r.src_loc_step), g["src_loc_step"])
    img = np.stack(r.get_results())
    for k in range(3):
        if np.abs(g["img"][k]).max() > 0:
            assert rel_l2(img[k], g["img"][k]) <= IMG_TOL, (k, rel_l2(img[k], g["img"][k]))
    r.cleanup()


def test_source_normalized_imaging_vs_fp64_oracle():
    """method="source_normalized" (extension): the cross-correlation image of
    each component divided by the source illumination sum_t snapshot^2 +
    eps * max, against the FP64 oracle; rel-L2 <= 1e-4.  The same through
    BatchedRTM.migrate's FP64 stack."""
    from oracle import fd_oracle
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    g = load_golden("fwbw_basic")
    c = _common(g)
    c.pop("surface_matrix_field")
    wav = dict(wavelet_u_field=g["wu"], wavelet_v_field=g["wv"], wavelet_w_field=g["ww"])
    isnap, eps = 3, 1e-3
    fm = ForwardModeling(isnap=isnap, **_fields(g, "s"), **c, **wav)
    assert fm.run(save=True) == 0
    bw = BackwardModeling(obsdata_u_field=g["obs"][0], obsdata_v_field=g["obs"][1], obsdata_w_field=g["obs"][2],
                          **_fields(g, "s"), **c)
    assert bw.run_calc(fm.u_save_field, fm.v_save_field, fm.w_save_field, fm.isnaps_field, fm.num_snaps, isnap,
                       method="source_normalized", normalization_eps=eps) == 0
    img = np.stack(bw.get_results())
    kw = dict(dx=float(g["dx"]), dz=float(g["dz"]), nt=int(g["nt"]), fs=float(g["fs"]), fw=int(g["fw"]))
    f = fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"],
                          rec=g["rec"], isnap=isnap, save=True, **kw)
    b = fd_oracle.backward(g["mu_s"], g["lam_s"], g["rho_s"], rec=g["rec"], ou=g["obs"][0], ov=g["obs"][1],
                           ow=g["obs"][2], snaps=f["snaps"], isnaps=f["isnaps"], num_snaps=f["num_snaps"],
                           isnap=isnap, **kw)
    slots = fd_oracle.imaging_slots(kw["nt"], isnap, f["isnaps"], f["num_snaps"])
    ref = fd_oracle.source_normalized(b["img"], f["snaps"], slots, eps)
    assert np.abs(ref).max() > 0
    e = rel_l2(img, ref)
    assert e <= IMG_TOL, e
    assert rel_l2(img, b["img"]) > 0.5  # the plain correlation is a different image
    # batched path: the FP64 stack of one full-window shot
    b2 = BatchedRTM(g["mu_s"], g["lam_s"], g["rho_s"], kw["dx"], kw["dz"], kw["fs"], kw["nt"], kw["fw"],
                    [ShotGeometry(0, c["nx"], g["src"], g["rec"])], modes=3, tune=None)
    w = np.stack([g["wu"], g["wv"], g["ww"]])
    _, _, st = b2.migrate(w, g["obs"], isnap=isnap, method="source_normalized", normalization_eps=eps)
    e2 = rel_l2(st.cpu().numpy(), ref)
    assert e2 <= IMG_TOL, e2
    b2.close()
