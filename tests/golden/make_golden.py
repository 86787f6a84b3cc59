"""Generate golden vectors by running the UNMODIFIED TaichiRTM reference source
(``src/forward_modeling.py``, ``src/backward_modeling.py``, ``src/rtm.py``)
under the NumPy Taichi stub in ``taichi_stub.py`` (FP64, serial, tiny grids).

Test infrastructure only.  Run where the reference is checked out, naming its
root in ``TAICHIRTM_REF`` (the directory that holds ``src/``):

    TAICHIRTM_REF=<path to TaichiRTM> python tests/golden/make_golden.py

Writes ``tests/golden/*.npz``.  The fixtures are committed; the GPU box never
needs the reference.
"""
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("TAICHIRTM_REF", "")


def load_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        raise SystemExit("set TAICHIRTM_REF to the TaichiRTM checkout (the directory holding src/)")
    os.environ.setdefault("TQDM_DISABLE", "1")
    sys.path.insert(0, HERE)
    import taichi_stub  # noqa: E402

    sys.modules["taichi"] = taichi_stub.as_module()
    src = os.path.join(REF, "src")
    spec = importlib.util.spec_from_file_location(
        "taichirtm_reference", os.path.join(src, "__init__.py"),
        submodule_search_locations=[src])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["taichirtm_reference"] = pkg
    spec.loader.exec_module(pkg)
    return pkg, sys.modules["taichi"]


def ricker(nt, dt, f0, t0=None):
    t = np.arange(nt) * dt
    t0 = 1.0 / f0 if t0 is None else t0
    a = (np.pi * f0 * (t - t0)) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def layered(nx, nz, seed, smooth=False):
    """Three flat layers, Vs = Vp/1.73, Gardner density (rho = 310 Vp^0.25)."""
    rng = np.random.default_rng(seed)
    vp = np.empty((nx, nz), np.float64)
    b1, b2 = nz // 3, 2 * nz // 3
    vp[:, :b1] = 1500.0
    vp[:, b1:b2] = 2500.0
    vp[:, b2:] = 3500.0
    vp *= 1.0 + 0.02 * rng.standard_normal((nx, nz))
    if smooth:
        k = np.array([0.25, 0.5, 0.25])
        for _ in range(3):
            vp = np.apply_along_axis(lambda r: np.convolve(np.pad(r, 1, mode="edge"), k, "valid"), 1, vp)
            vp = np.apply_along_axis(lambda r: np.convolve(np.pad(r, 1, mode="edge"), k, "valid"), 0, vp)
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    mu = (rho * vs ** 2).astype(np.float32)
    lam = (rho * vp ** 2 - 2.0 * mu).astype(np.float32)
    return mu, lam, rho.astype(np.float32)


def fields_from(ti, arrs, dtype):
    out = []
    for a in arrs:
        f = ti.field(dtype=dtype, shape=a.shape)
        f.from_numpy(a)
        out.append(f)
    return out


def run_fw_bw(pkg, ti, *, nx, nz, dx, dz, nt, fs, fw, src, wav, rec, isnap,
              surface=None, seed=0):
    """Forward on the true model (observed data), forward with snapshots on
    the smoothed model, backward on the smoothed model with the observed
    data.  Returns a dict of inputs and outputs."""
    mu_t, lam_t, rho_t = layered(nx, nz, seed)
    mu_s, lam_s, rho_s = layered(nx, nz, seed, smooth=True)
    src = np.asarray(src, np.int32)
    rec = np.asarray(rec, np.int32)
    wu, wv, ww = [np.asarray(w, np.float32) for w in wav]
    src_f, rec_f = fields_from(ti, [src, rec], ti.i32)
    wu_f, wv_f, ww_f = fields_from(ti, [wu, wv, ww], ti.f32)
    sm_f = None
    if surface is not None:
        (sm_f,) = fields_from(ti, [surface.astype(np.float32)], ti.f32)

    def fwd(mu, lam, rho, save):
        m_f = fields_from(ti, [mu, lam, rho], ti.f32)
        fm = pkg.ForwardModeling(
            nx=nx, nz=nz, dx=dx, dz=dz, nt=nt, fs=fs, mu_field=m_f[0], lam_field=m_f[1],
            rho_field=m_f[2], absorbing_frame=fw, src_loc_field=src_f,
            wavelet_u_field=wu_f, wavelet_v_field=wv_f, wavelet_w_field=ww_f,
            recv_loc_field=rec_f, isnap=isnap, surface_matrix_field=sm_f,
            num_sources=len(src), num_receivers=len(rec))
        flag = fm.run(save=save)
        return fm, m_f, flag

    t0 = time.time()
    fm_t, _, flag_t = fwd(mu_t, lam_t, rho_t, False)
    obs = fm_t.get_seismogram()
    fm_s, m_s, flag_s = fwd(mu_s, lam_s, rho_s, True)
    syn = fm_s.get_seismogram()
    obs_f = fields_from(ti, list(obs), ti.f32)
    bm = pkg.BackwardModeling(
        nx=nx, nz=nz, dx=dx, dz=dz, nt=nt, fs=fs, mu_field=m_s[0], lam_field=m_s[1],
        rho_field=m_s[2], absorbing_frame=fw, src_loc_field=src_f,
        obsdata_u_field=obs_f[0], obsdata_v_field=obs_f[1], obsdata_w_field=obs_f[2],
        recv_loc_field=rec_f, surface_matrix_field=sm_f,
        num_sources=len(src), num_receivers=len(rec))
    flag_b = bm.run_calc(fm_s.u_save_field, fm_s.v_save_field, fm_s.w_save_field,
                         fm_s.isnaps_field, fm_s.num_snaps, isnap)
    img = bm.get_results()
    print(f"  fw/fw/bw done in {time.time() - t0:.1f}s")
    return dict(
        nx=nx, nz=nz, dx=dx, dz=dz, nt=nt, fs=fs, fw=fw, isnap=isnap,
        src=src, rec=rec, wu=wu, wv=wv, ww=ww,
        surface=(surface.astype(np.float32) if surface is not None else np.zeros((0, 0), np.float32)),
        mu_t=mu_t, lam_t=lam_t, rho_t=rho_t, mu_s=mu_s, lam_s=lam_s, rho_s=rho_s,
        obs=np.stack(obs), syn=np.stack(syn),
        snaps=np.stack([fm_s.u_save_field.to_numpy(), fm_s.v_save_field.to_numpy(),
                        fm_s.w_save_field.to_numpy()]),
        isnaps=fm_s.isnaps_field.to_numpy(), num_snaps=fm_s.num_snaps,
        absorb=fm_s.absorb_coeff.to_numpy(),
        mxz=fm_s.mxz.to_numpy(), myx=fm_s.myx.to_numpy(), myz=fm_s.myz.to_numpy(),
        inv_rho=fm_s.inv_rho.to_numpy(), inv_rho_u=fm_s.inv_rho_u.to_numpy(),
        inv_rho_w=fm_s.inv_rho_w.to_numpy(),
        img=np.stack(img), flags=np.array([flag_t, flag_s, flag_b]))


def case_basic(pkg, ti):
    nx, nz, nt, fs = 36, 28, 160, 2000.0
    w = ricker(nt, 1.0 / fs, 60.0)
    src = [[18, 2], [9, 5]]
    wav = (np.stack([0.3 * w, 0.0 * w]), np.stack([0.5 * w, 0.2 * w]), np.stack([w, 0.7 * w]))
    rec = [[i, 1] for i in range(0, nx, 3)] + [[nx - 1, 1], [20, 10], [20, 10]]
    return run_fw_bw(pkg, ti, nx=nx, nz=nz, dx=5.0, dz=5.0, nt=nt, fs=fs, fw=7,
                     src=src, wav=wav, rec=rec, isnap=3, seed=11)


def case_topo(pkg, ti):
    nx, nz, nt, fs = 32, 24, 120, 2000.0
    w = ricker(nt, 1.0 / fs, 60.0)
    surface = np.ones((nx, nz), np.float32)
    for i in range(nx):
        surface[i, : (i // 8)] = 0.0
    src = [[16, 4]]
    wav = (0.0 * w[None], 0.5 * w[None], w[None])
    rec = [[i, 1 + i // 8] for i in range(1, nx - 1, 2)]
    return run_fw_bw(pkg, ti, nx=nx, nz=nz, dx=4.0, dz=5.0, nt=nt, fs=fs, fw=6,
                     src=src, wav=wav, rec=rec, isnap=4, surface=surface, seed=12)


def case_narrow(pkg, ti):
    # nx < 2*FW: the left/right sponge strips overlap and the right strip's
    # writes win (forward_modeling.py:214-235 run in order).
    nx, nz, nt, fs = 14, 26, 90, 2500.0
    w = ricker(nt, 1.0 / fs, 80.0)
    src = [[7, 3]]
    wav = (w[None], 0.4 * w[None], 0.8 * w[None])
    rec = [[i, 1] for i in range(nx)]
    return run_fw_bw(pkg, ti, nx=nx, nz=nz, dx=3.0, dz=3.0, nt=nt, fs=fs, fw=9,
                     src=src, wav=wav, rec=rec, isnap=1, seed=13)


def case_edge_source(pkg, ti):
    # A source on an edge cell multiplies by inv_rho_u = 1/0 = inf
    # (forward_modeling.py:291-307, 437-443): the wavefield becomes inf/NaN.
    nx, nz, nt, fs = 20, 16, 30, 2000.0
    w = ricker(nt, 1.0 / fs, 60.0)
    src = [[0, 4]]
    wav = (w[None], w[None], w[None])
    rec = [[i, 1] for i in range(0, nx, 2)]
    return run_fw_bw(pkg, ti, nx=nx, nz=nz, dx=5.0, dz=5.0, nt=nt, fs=fs, fw=4,
                     src=src, wav=wav, rec=rec, isnap=2, seed=14)


def case_rtm(pkg, ti, *, v_fix, heights):
    """ReverseTimeMigration.run end to end (rtm.py:846-1029) on a tiny survey."""
    nt, fs = 70, 1000.0
    rng = np.random.default_rng(21)
    nrec = 5
    rec_x = np.linspace(0.0, 1.6, nrec).astype(np.float32)
    w = ricker(nt, 1.0 / fs, 50.0)
    obs = (0.01 * rng.standard_normal((3, nrec, nt))).astype(np.float32)
    obs[2, :, 5:25] += w[None, :20] * 0.1
    r = pkg.ReverseTimeMigration()
    r.set_observed_data(obs[0], obs[1], obs[2]).set_source(0 * w, 0.3 * w, w, 0.8)
    r.set_receivers(rec_x).set_frequency(fs).set_boundary(3)
    r.set_velocity_range(40.0, 200.0, 6).set_poisson_ratio(0.2)
    if v_fix is not None:
        r.fix_velocity(v_fix)
    if heights is not None:
        r.set_topography(heights)
    t0 = time.time()
    r.run()
    print(f"  rtm.run done in {time.time() - t0:.1f}s")
    sm = getattr(r, "surface_matrix", None)
    return dict(
        obs=obs, src_w=np.stack([0 * w, 0.3 * w, w]), src_x=np.float64(0.8), rec_x=rec_x,
        fs=fs, fw=3, vmin=40.0, vmax=200.0, vstep=6, poisson=0.2, rho=1500.0,
        v_fix=np.float64(np.nan if v_fix is None else v_fix),
        heights=(np.asarray(heights, np.float32) if heights is not None else np.zeros(0, np.float32)),
        img=np.stack(r.get_results()), dx=r.dx, nx=r.nx, nz=r.nz, cfl=r.CFL,
        src_loc_step=np.asarray(r.src_loc_step), offset=r.offset,
        surface=(sm if sm is not None else np.zeros((0, 0), np.float32)))


def main():
    pkg, ti = load_reference()
    cases = {
        "fwbw_basic": lambda: case_basic(pkg, ti),
        "fwbw_topo": lambda: case_topo(pkg, ti),
        "fwbw_narrow": lambda: case_narrow(pkg, ti),
        "fwbw_edge_source": lambda: case_edge_source(pkg, ti),
        "rtm_vfix": lambda: case_rtm(pkg, ti, v_fix=100.0, heights=None),
        "rtm_vscan_topo": lambda: case_rtm(pkg, ti, v_fix=None,
                                            heights=np.array([0.0, -0.5, -1.0, -0.7, -0.2])),
    }
    only = sys.argv[1:]
    for name, fn in cases.items():
        if only and name not in only:
            continue
        print(name)
        out = fn()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


if __name__ == "__main__":
    main()
