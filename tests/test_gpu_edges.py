"""Edge cases of the propagation entry points, bit-exact against the NumPy
FP32 restatement (same one-time FP64 set-up, Kahan imaging):

* a shot without sources and a shot without receivers;
* the smallest grid (3 x 3: one interior cell) and no sponge (FW = 0);
* time axes of 1, 2, 3 and 7 steps (odd last steps with two steps per launch);
* shot windows touching the first and the last model row, batched, with one
  and two steps per launch, equal to standalone runs on the cropped models.
"""
import numpy as np
import pytest
import torch

from oracle import fd_oracle

pytestmark = pytest.mark.gpu


def _model(nx, nz, seed=1):
    rng = np.random.default_rng(seed)
    vp = 2000.0 + 600.0 * rng.random((nx, nz))
    vs, rho = vp / 1.8, 310.0 * vp ** 0.25
    mu = (rho * vs ** 2).astype(np.float32)
    lam = (rho * vp ** 2 - 2 * rho * vs ** 2).astype(np.float32)
    return mu, lam, rho.astype(np.float32)


def _ricker(nt, fs=2000.0, f0=80.0, t0=0.01):
    t = np.arange(nt) / fs - t0
    a = (np.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _gpu_vs_restatement(nx, nz, nt, fw, src, rec, wav, isnap, tune):
    """Forward with snapshots and backward with imaging on the GPU and in the
    FP32 restatement; returns both results."""
    from taichirtm_b200.plan import Plan, ShotGeometry
    mu, lam, rho = _model(nx, nz)
    kw = dict(dx=4.0, dz=4.0, nt=nt, fs=2000.0, fw=fw)
    wav = np.ascontiguousarray(wav[:, :len(src)])
    ref = fd_oracle.forward(mu, lam, rho, src=src, wu=wav[0], wv=wav[1], ww=wav[2], rec=rec, isnap=isnap, save=True,
                            dtype=np.float32, setup_f64=True, **kw)
    obs = (ref["seis"] * 0.5 + 1e-3).astype(np.float32) if len(rec) else np.zeros((3, 0, nt), np.float32)
    bref = fd_oracle.backward(mu, lam, rho, rec=rec, ou=obs[0], ov=obs[1], ow=obs[2], snaps=ref["snaps"],
                              isnaps=ref["isnaps"], num_snaps=ref["num_snaps"], isnap=isnap, dtype=np.float32,
                              setup_f64=True, kahan=True, **kw)
    p = Plan(nx, nz, kw["dx"], kw["dz"], nt, kw["fs"], fw, 3, [ShotGeometry(0, nx, src, rec)], tune=tune)
    p.set_model(mu, lam, rho)
    f, seis, snaps, isn = p.forward(torch.as_tensor(wav), save=True, isnap=isnap)
    f2, img, _ = p.backward(torch.as_tensor(obs), snaps, isn, len(isn), isnap)
    out = dict(flag=int(f[0]), flag_b=int(f2[0]), seis=seis.cpu().numpy(), img=img.cpu().numpy(),
               snaps=[p.snapshot_view(snaps[c], len(isn)).cpu().numpy() for c in range(3)])
    p.close()
    return out, ref, bref


@pytest.mark.parametrize("tune", [dict(vec=2, rows=4, warps=2, tsteps=1), dict(vec=2, rows=4, warps=2, tsteps=2)])
@pytest.mark.parametrize("case", ["no_sources", "no_receivers"])
def test_shot_without_sources_or_receivers(case, tune):
    nx, nz, nt = 40, 36, 50
    src = np.zeros((0, 2), np.int32) if case == "no_sources" else np.array([[20, 5]], np.int32)
    rec = np.zeros((0, 2), np.int32) if case == "no_receivers" else np.array([[i, 1] for i in range(3, 37, 3)], np.int32)
    wav = np.zeros((3, max(len(src), 1), nt), np.float32)
    wav[:, 0] = _ricker(nt)[None]
    g, ref, bref = _gpu_vs_restatement(nx, nz, nt, 6, src, rec, wav, 4, tune)
    assert g["flag"] == 0 and g["flag_b"] == 0
    assert g["seis"].shape == (3, len(rec), nt)
    assert np.array_equal(g["seis"], ref["seis"])
    for c in range(3):
        assert np.array_equal(g["snaps"][c], ref["snaps"][c])
    assert np.array_equal(g["img"], bref["img"])
    if case == "no_sources":
        assert np.abs(g["snaps"][2]).max() == 0.0   # nothing excites the forward wavefield
    else:
        assert np.abs(g["snaps"][2]).max() > 0.0 and np.abs(g["img"]).max() == 0.0


@pytest.mark.parametrize("tune", [dict(vec=1, rows=1, warps=1, prefetch=0), dict(vec=2, rows=2, warps=1, tsteps=2),
                                  dict(vec=4, rows=8, warps=4, prefetch=3), dict(vec=2, rows=2, warps=3, tsteps=2, prefetch=3),
                                  dict(vec=4, rows=3, warps=1, tsteps=2, prefetch=4)])
@pytest.mark.parametrize("grid", [(3, 3, 0), (5, 4, 0), (23, 17, 0), (23, 17, 4)])
def test_smallest_grids_and_no_sponge(grid, tune):
    nx, nz, fw = grid
    nt = 40
    src = np.array([[nx // 2, nz // 2]], np.int32)
    rec = np.array([[i, j] for i in range(nx) for j in (0, nz // 2, nz - 1)], np.int32)
    wav = np.zeros((3, 1, nt), np.float32)
    wav[:, 0] = _ricker(nt)[None] * np.array([[0.3], [0.6], [1.0]], np.float32)
    g, ref, bref = _gpu_vs_restatement(nx, nz, nt, fw, src, rec, wav, 3, tune)
    assert g["flag"] == ref["flag"] == 0
    assert np.array_equal(g["seis"], ref["seis"])
    for c in range(3):
        assert np.array_equal(g["snaps"][c], ref["snaps"][c])
    assert np.array_equal(g["img"], bref["img"])
    assert np.abs(g["seis"]).max() > 0


@pytest.mark.parametrize("tune", [dict(vec=2, rows=4, warps=2, tsteps=1), dict(vec=2, rows=5, warps=1, tsteps=2, prefetch=4),
                                  dict(vec=4, rows=3, warps=1, tsteps=2, prefetch=4)])
@pytest.mark.parametrize("nt,isnap", [(1, 1), (2, 1), (3, 2), (7, 3)])
def test_short_and_odd_time_axes(nt, isnap, tune):
    """Time axes of 1, 2, 3 and 7 steps: an odd last step with two steps
    per launch, no imaging step at all (nt 1), bit-exact against the FP32
    restatement."""
    nx, nz = 30, 24
    src = np.array([[15, 5]], np.int32)
    rec = np.array([[i, 2] for i in range(2, 28, 2)] + [[15, 5], [14, 5], [16, 5], [15, 4], [15, 6], [13, 7]],
                   np.int32)  # a line, and cells at and around the source
    wav = np.zeros((3, 1, nt), np.float32)
    wav[:, 0, 0] = np.array([0.3, 0.6, 1.0], np.float32)
    if nt > 1:
        wav[:, 0, 1] = np.array([-0.1, 0.2, -0.5], np.float32)
    g, ref, bref = _gpu_vs_restatement(nx, nz, nt, 4, src, rec, wav, isnap, tune)
    assert g["flag"] == ref["flag"] == 0
    assert np.array_equal(g["seis"], ref["seis"])
    for c in range(3):
        assert np.array_equal(g["snaps"][c], ref["snaps"][c])
    assert np.array_equal(g["img"], bref["img"])
    assert np.abs(g["seis"]).max() > 0


@pytest.mark.parametrize("tsteps,prefetch", [(1, 1), (2, 1), (2, 3)])
def test_windows_touching_the_model_edges(tsteps, prefetch):
    """Windows [0, 40), [60, 100) (the last rows) and [0, 100) in one batched
    plan equal standalone runs on the cropped models, bit for bit."""
    from taichirtm_b200.plan import Plan, ShotGeometry
    nx, nz, nt, fw = 100, 70, 60, 8
    mu, lam, rho = _model(nx, nz, seed=4)
    wins = [(0, 40), (60, 40), (0, 100)]
    shots, wav = [], []
    for x0, w in wins:
        src = np.array([[w // 2, 3], [1, 2], [w - 2, 5]], np.int32)  # sources next to the window edges
        rec = np.array([[i, 1] for i in range(w)] + [[0, 30], [w - 1, 30]], np.int32)
        shots.append(ShotGeometry(x0, w, src, rec))
        wv = np.zeros((3, 3, nt), np.float32)
        wv[:, :] = _ricker(nt)[None, None]
        wav.append(wv)
    tune = dict(vec=2, rows=3, warps=2, tsteps=tsteps, prefetch=prefetch)
    p = Plan(nx, nz, 4.0, 4.0, nt, 2000.0, fw, 1, shots, tune=tune)
    p.set_model(mu, lam, rho)
    f, seis, _, _ = p.forward(torch.as_tensor(np.concatenate(wav, axis=1)))
    seis = seis.cpu().numpy()
    p.close()
    r0 = 0
    for (x0, w), sh, wv in zip(wins, shots, wav):
        q = Plan(w, nz, 4.0, 4.0, nt, 2000.0, fw, 1, [ShotGeometry(0, w, sh.src, sh.rec)], tune=tune)
        q.set_model(*(np.ascontiguousarray(a[x0:x0 + w]) for a in (mu, lam, rho)))
        _, s1, _, _ = q.forward(torch.as_tensor(wv))
        q.close()
        n = len(sh.rec)
        assert np.array_equal(seis[:, r0:r0 + n], s1.cpu().numpy())
        r0 += n
    assert int(f.max()) == 0


@pytest.mark.parametrize("checkpoint", [None, dict(every=9, dtype="f32")])
def test_migrate_with_pinned_host_observed_data(checkpoint):
    """BatchedRTM.migrate copies pinned host observed data on a side stream
    while the forward pass runs; the stack equals the one from device data."""
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    nx, nz, nt, fw = 90, 60, 70, 8
    mu, lam, rho = _model(nx, nz, seed=6)
    shots = [ShotGeometry(0, 50, np.array([[25, 3]], np.int32), np.array([[i, 1] for i in range(50)], np.int32)),
             ShotGeometry(40, 50, np.array([[25, 3]], np.int32), np.array([[i, 1] for i in range(0, 50, 2)], np.int32))]
    wav = np.zeros((3, 2, nt), np.float32)
    wav[2] = _ricker(nt)[None]
    b = BatchedRTM(mu, lam, rho, 4.0, 4.0, 2000.0, nt, fw, shots, tune=dict(vec=2, rows=8, warps=2, tsteps=2))
    _, seis, _, _ = b.forward(wav)
    obs_dev = (seis * 0.8).contiguous()
    obs_host = obs_dev.cpu().pin_memory()
    _, _, st_dev = b.migrate(wav, obs_dev, isnap=4, checkpoint=checkpoint)
    _, _, st_host = b.migrate(wav, obs_host, isnap=4, checkpoint=checkpoint)
    assert np.abs(st_dev.cpu().numpy()).max() > 0
    assert torch.equal(st_dev, st_host)
    b.close()
