"""Parity at the benchmark sizes, through properties that do not depend on size.

* The 64-shot batched P-SV workload (2001 x 801) runs bit-identically with one
  and with two time steps per launch.
* Its FP64 stack equals, bit for bit, the sum of the same shots run one by
  one in their own plans, added in the same order.
* One shot of that workload at full length (nt 3000, isnap 16) against the
  FP64 C restatement: seismogram rel-L2 <= 1e-5, image rel-L2 <= 1e-4.
* A full-width shot on the 4001 x 1601 model against the FP64 C restatement
  over a shortened time axis: seismogram rel-L2 <= 1e-5.
"""
import numpy as np
import pytest
import torch

from oracle import c_oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
IMG_TOL = 1e-4


def _c3(nt):
    from taichirtm_b200 import synthetic as S
    return S.config3(nt=nt)


def _migrate(sv, shots_idx, tune, stack=None, graphs=True):
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    sub = [sv.shots[i] for i in shots_idx]
    geo = [ShotGeometry(s.x0, s.nx, s.src, s.rec) for s in sub]
    wav = np.concatenate([s.wavelets for s in sub], axis=1)
    mu, lam, rho = sv.material(migration=True)
    b = BatchedRTM(mu, lam, rho, sv.dx, sv.dz, sv.fs, sv.nt, sv.fw, geo, tune=tune, graphs=graphs)
    ff, seis, _, _ = b.forward(wav, check_interval=100)
    obs = (seis * 0.5).contiguous()
    _, _, st = b.migrate(wav, obs, isnap=16, check_interval=100, stack=stack)
    out = (seis.cpu().numpy(), st)
    b.close()
    return out


def test_full_batch_one_and_two_steps_per_launch_bit_identical():
    sv = _c3(120)
    idx = list(range(len(sv.shots)))
    s1, st1 = _migrate(sv, idx, dict(vec=2, rows=32, warps=1, tsteps=1))
    s2, st2 = _migrate(sv, idx, dict(vec=2, rows=32, warps=1, tsteps=2))
    assert len(idx) == 64 and np.abs(st1.cpu().numpy()).max() > 0
    assert np.array_equal(s1, s2)
    assert torch.equal(st1, st2)


def test_full_size_stack_equals_sum_of_standalone_shots():
    sv = _c3(120)
    idx = [0, 21, 42, 63]
    tune = dict(vec=2, rows=16, warps=2, tsteps=2)
    _, batched = _migrate(sv, idx, tune)
    acc = torch.zeros_like(batched)
    for i in idx:  # same shot order: the FP64 additions happen in the same sequence
        _migrate(sv, [i], tune, stack=acc)
    assert torch.equal(batched, acc)


def test_full_length_batched_shot_vs_fp64_oracle():
    """Shot 0 of the batched workload (582 x 801 window, nt 3000, isnap 16),
    migrated through BatchedRTM, against the FP64 C restatement run on the
    cropped model."""
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    sv = _c3(3000)
    sh = sv.shots[0]
    mu, lam, rho = sv.material(migration=True)
    crop = [np.ascontiguousarray(x[sh.x0:sh.x0 + sh.nx]) for x in (mu, lam, rho)]
    kw = dict(dx=sv.dx, dz=sv.dz, nt=sv.nt, fs=sv.fs, fw=sv.fw, dtype=np.float64, modes=1)
    f = c_oracle.forward(*crop, src=sh.src, wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2],
                         rec=sh.rec, save=True, isnap=16, **kw)
    obs = (f["seis"] * 0.5).astype(np.float32)
    b = c_oracle.backward(*crop, rec=sh.rec, obs=obs, snaps=f["snaps"], isnaps=f["isnaps"],
                          num_snaps=f["num_snaps"], isnap=16, **kw)
    r = BatchedRTM(mu, lam, rho, sv.dx, sv.dz, sv.fs, sv.nt, sv.fw, [ShotGeometry(sh.x0, sh.nx, sh.src, sh.rec)],
                   tune=dict(vec=2, rows=32, warps=1, tsteps=2))
    ff, seis, _, _ = r.forward(sh.wavelets)
    assert int(ff.max()) == 0
    assert rel_l2(seis.cpu().numpy()[[0, 2]], f["seis"][[0, 2]]) <= SEIS_TOL
    _, fb, st = r.migrate(sh.wavelets, obs, isnap=16)
    assert int(fb.max()) == 0
    img = st.cpu().numpy()[:, sh.x0:sh.x0 + sh.nx]
    e = rel_l2(img[[0, 2]], b["img"][[0, 2]])
    print(f"batched-workload shot 0 at full length vs FP64: seismograms "
          f"{rel_l2(seis.cpu().numpy()[[0, 2]], f['seis'][[0, 2]]):.2e}, image {e:.2e}")
    assert e <= IMG_TOL, e
    r.close()


def test_largest_grid_full_width_shot_vs_fp64_oracle():
    """A shot covering the whole 4001 x 1601 model (6.4 M cells), 120 steps."""
    from taichirtm_b200 import synthetic as S
    from taichirtm_b200.plan import Plan, ShotGeometry
    sv = S.config5(nt=120)
    mu, lam, rho = sv.material()
    nx, nz, nt = sv.nx, sv.nz, sv.nt
    t = np.arange(nt) / sv.fs - 0.02
    a = (np.pi * 60.0 * t) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.array([[nx // 2, 2]], np.int32)
    rec = np.stack([np.arange(nx // 2 - 300, nx // 2 + 300), np.ones(600, int)], 1).astype(np.int32)
    wav = np.zeros((3, 1, nt), np.float32)
    wav[0, 0], wav[2, 0] = 0.5 * w, w
    ref = c_oracle.forward(mu, lam, rho, dx=sv.dx, dz=sv.dz, nt=nt, fs=sv.fs, fw=sv.fw, src=src, wu=wav[0, 0],
                           wv=wav[1, 0], ww=wav[2, 0], rec=rec, dtype=np.float64, modes=1)
    p = Plan(nx, nz, sv.dx, sv.dz, nt, sv.fs, sv.fw, 1, [ShotGeometry(0, nx, src, rec)],
             tune=dict(vec=2, rows=32, warps=1, tsteps=2))
    p.set_model(mu, lam, rho)
    ff, seis, _, _ = p.forward(torch.as_tensor(wav))
    assert int(ff.max()) == 0
    s = seis.cpu().numpy()
    assert np.abs(s).max() > 0
    e = rel_l2(s[[0, 2]], ref["seis"][[0, 2]])
    assert e <= SEIS_TOL, e
    p.close()
