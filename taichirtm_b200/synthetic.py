"""Seeded synthetic surveys with the shapes of the five benchmark workloads.

No public dataset exists for this path, so benchmarks and parity tests run on
these generators.  Conventions (grid index i = x, j = z; arrays (nx, nz), z
fastest, like the reference's fields):

  * Gardner density rho = 310 * Vp**0.25 (SI), Vs = Vp / 1.73 unless stated.
  * Ricker wavelet (1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2), tau = t - 1/f.
  * Material as the reference builds it (src/rtm.py:901-902):
    mu = rho vs^2, lam = rho vp^2 - 2 mu.
  * Receivers at j = 1, sources at j = 2 (src/rtm.py:674-676 put both at 1;
    the source depth here follows the workload description).
  * Seeds: numpy.random.default_rng(config number), 100 + config number for
    per-shot draws.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


def ricker(nt, dt, f0):
    t = np.arange(nt, dtype=np.float64) * dt
    a = (np.pi * f0 * (t - 1.0 / f0)) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def gaussian_smooth(a, sigma):
    """Separable Gaussian smoothing (reflecting edges), sigma in cells."""
    if sigma <= 0:
        return np.array(a, dtype=np.float64, copy=True)
    r = int(np.ceil(3.0 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = np.asarray(a, np.float64)
    for ax in range(out.ndim):
        pad = [(0, 0)] * out.ndim
        pad[ax] = (r, r)
        p = np.pad(out, pad, mode="reflect")
        acc = np.zeros_like(out)
        for q in range(2 * r + 1):
            sl = [slice(None)] * out.ndim
            sl[ax] = slice(q, q + out.shape[ax])
            acc += k[q] * p[tuple(sl)]
        out = acc
    return out


def gardner(vp):
    return 310.0 * np.asarray(vp, np.float64) ** 0.25


def lame(vp, vs, rho):
    vp, vs, rho = (np.asarray(x, np.float64) for x in (vp, vs, rho))
    mu = rho * vs ** 2
    lam = rho * vp ** 2 - 2.0 * mu
    return mu.astype(np.float32), lam.astype(np.float32), rho.astype(np.float32)


def add_anomalies(v, rng, n, amp=0.15, sig=(10.0, 40.0)):
    nx, nz = v.shape
    ii, jj = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    scale = np.ones_like(v, dtype=np.float64)
    for _ in range(n):
        ci, cj = rng.uniform(0, nx), rng.uniform(0, nz)
        a = rng.uniform(-amp, amp)
        s = rng.uniform(*sig)
        scale *= 1.0 + a * np.exp(-((ii - ci) ** 2 + (jj - cj) ** 2) / (2.0 * s * s))
    return v * scale


def layered_vp(nx, nz, speeds):
    vp = np.empty((nx, nz), np.float64)
    edges = np.linspace(0, nz, len(speeds) + 1).astype(int)
    for k, s in enumerate(speeds):
        vp[:, edges[k]:edges[k + 1]] = s
    return vp


@dataclass
class Shot:
    """One shot on a window of the global model: rows [x0, x0 + nx) of it."""
    x0: int
    nx: int
    src: np.ndarray            # (nsrc, 2) int32, LOCAL grid indices
    rec: np.ndarray            # (nrec, 2) int32, LOCAL grid indices
    wavelets: np.ndarray       # (3, nsrc, nt) float32 (u, v, w)


@dataclass
class Survey:
    name: str
    nx: int
    nz: int
    dx: float
    dz: float
    fs: float
    nt: int
    fw: int
    mode: str                  # "psv", "sh" or "both"
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    vp_mig: Optional[np.ndarray] = None
    vs_mig: Optional[np.ndarray] = None
    rho_mig: Optional[np.ndarray] = None
    shots: List[Shot] = field(default_factory=list)

    @property
    def dt(self):
        return 1.0 / self.fs

    def material(self, migration=False):
        if migration and self.vp_mig is not None:
            return lame(self.vp_mig, self.vs_mig, self.rho_mig)
        return lame(self.vp, self.vs, self.rho)

    def cells(self):
        return sum(s.nx for s in self.shots) * self.nz


def _full_width_shot(nx, src_i, src_j, nt, dt, f0, comp, rec_j=1, rec=None):
    w = ricker(nt, dt, f0)
    wav = np.zeros((3, 1, nt), np.float32)
    wav[comp, 0] = w
    if rec is None:
        rec = np.stack([np.arange(nx), np.full(nx, rec_j)], 1)
    return Shot(0, nx, np.array([[src_i, src_j]], np.int32), np.asarray(rec, np.int32), wav)


def config1(nt=2000):
    """Plain P-SV RTM, one shot: 301 x 151, dx = dz = 5 m, dt = 0.5 ms, three
    flat layers (Vp 1500/2500/3500), Vs = Vp/1.73, Gardner density, migration
    model = Gaussian-smoothed copy (sigma 5 cells), FW 40, Ricker 20 Hz
    vertical force at (150, 2), 301 receivers at j = 1."""
    nx, nz = 301, 151
    vp = np.empty((nx, nz))
    vp[:, :50], vp[:, 50:100], vp[:, 100:] = 1500.0, 2500.0, 3500.0
    vs, rho = vp / 1.73, gardner(vp)
    vpm = gaussian_smooth(vp, 5.0)
    s = Survey("c1_psv_rtm", nx, nz, 5.0, 5.0, 2000.0, nt, 40, "psv", vp, vs, rho,
               vpm, vpm / 1.73, gardner(vpm))
    s.shots = [_full_width_shot(nx, 150, 2, nt, s.dt, 20.0, comp=2)]
    return s


def config2(nt=4000):
    """Plain SH RTM, one shot: 1001 x 501, dx = dz = 4 m, dt = 0.4 ms; Vs
    linear 800-2400 m/s with 20 seeded Gaussian anomalies (+-15 %, sigma
    10-40 cells), Vp = 1.73 Vs, Gardner density, FW 50, Ricker 15 Hz point
    force on v at (500, 2), 1001 receivers at j = 1."""
    nx, nz = 1001, 501
    rng = np.random.default_rng(2)
    vs = np.broadcast_to(800.0 + 1600.0 * np.arange(nz) / (nz - 1), (nx, nz)).copy()
    vs = add_anomalies(vs, rng, 20)
    vp = 1.73 * vs
    rho = gardner(vp)
    vsm = gaussian_smooth(vs, 10.0)
    s = Survey("c2_sh_rtm", nx, nz, 4.0, 4.0, 2500.0, nt, 50, "sh", vp, vs, rho,
               1.73 * vsm, vsm, gardner(1.73 * vsm))
    s.shots = [_full_width_shot(nx, 500, 2, nt, s.dt, 15.0, comp=1)]
    return s


def _windowed_shots(nx, centres, counts, fw, nt, dt, f0, src_j=2, rec_j=1):
    shots = []
    w = ricker(nt, dt, f0)
    for c, n in zip(centres, counts):
        r0 = max(0, c - n // 2)
        r1 = min(nx, r0 + n)
        r0 = max(0, r1 - n)
        x0 = max(0, min(r0, c) - fw)
        x1 = min(nx, max(r1, c + 1) + fw)
        rec = np.stack([np.arange(r0, r1) - x0, np.full(r1 - r0, rec_j)], 1).astype(np.int32)
        wav = np.zeros((3, 1, nt), np.float32)
        wav[2, 0] = w
        shots.append(Shot(x0, x1 - x0, np.array([[c - x0, src_j]], np.int32), rec, wav))
    return shots


def config3(nt=3000, nshots=64):
    """Batched P-SV RTM: 2001 x 801, dx = 5 m, dt = 0.5 ms; four flat layers
    plus 20 seeded anomalies; 64 shots at i = 55 + 30 k; shot k records on
    U{200..800} contiguous receivers centred on it; shot window = receivers
    and source +- a 50-cell sponge."""
    nx, nz, fw = 2001, 801, 50
    rng = np.random.default_rng(3)
    vp = add_anomalies(layered_vp(nx, nz, [1500.0, 2200.0, 2900.0, 3600.0]), rng, 20)
    vs, rho = vp / 1.73, gardner(vp)
    vpm = gaussian_smooth(vp, 10.0)
    s = Survey("c3_batched_psv_rtm", nx, nz, 5.0, 5.0, 2000.0, nt, fw, "psv", vp, vs, rho,
               vpm, vpm / 1.73, gardner(vpm))
    counts = np.random.default_rng(103).integers(200, 801, size=nshots)
    centres = [55 + 30 * k for k in range(nshots)]
    s.shots = _windowed_shots(nx, centres, counts, fw, nt, s.dt, 20.0)
    return s


def config4(nt=3000, nshots=8):
    """FWI gradient: 1201 x 401, dx = 5 m, dt = 0.5 ms, 8 evenly spaced
    full-spread shots; true model = layers + seeded anomalies, starting model
    = Gaussian smoothing (sigma 15 cells) of it."""
    nx, nz, fw = 1201, 401, 50
    rng = np.random.default_rng(4)
    vp = add_anomalies(layered_vp(nx, nz, [1600.0, 2300.0, 3000.0]), rng, 12)
    vs, rho = vp / 1.73, gardner(vp)
    vpm = gaussian_smooth(vp, 15.0)
    s = Survey("c4_fwi_gradient", nx, nz, 5.0, 5.0, 2000.0, nt, fw, "psv", vp, vs, rho,
               vpm, gaussian_smooth(vs, 15.0), gaussian_smooth(rho, 15.0))
    centres = np.linspace(fw + 10, nx - fw - 10, nshots).astype(int)
    s.shots = [_full_width_shot(nx, c, 2, nt, s.dt, 15.0, comp=2) for c in centres]
    return s


def config5(nt=8000, nshots=32):
    """Large batched, checkpointed P-SV RTM: 4001 x 1601, dx = 5 m,
    dt = 0.4 ms, 32 shots each with U{1000..2000} receivers (seed 105)."""
    nx, nz, fw = 4001, 1601, 50
    rng = np.random.default_rng(5)
    vp = add_anomalies(layered_vp(nx, nz, [1500.0, 2200.0, 2900.0, 3600.0]), rng, 30)
    vs, rho = vp / 1.73, gardner(vp)
    vpm = gaussian_smooth(vp, 10.0)
    s = Survey("c5_large_batched", nx, nz, 5.0, 5.0, 2500.0, nt, fw, "psv", vp, vs, rho,
               vpm, vpm / 1.73, gardner(vpm))
    counts = np.random.default_rng(105).integers(1000, 2001, size=nshots)
    centres = np.linspace(fw + 600, nx - fw - 600, nshots).astype(int)
    s.shots = _windowed_shots(nx, centres, counts, fw, nt, s.dt, 20.0)
    return s


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}
