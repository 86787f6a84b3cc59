"""Vectorised NumPy restatement of TaichiRTM's 2-D elastic O(2,2) staggered-grid
propagators -- TEST INFRASTRUCTURE (the oracle), never the product.

Arrays use the reference's (nx, nz) layout, z fastest.  Every operation keeps
the reference's operand order so that an FP64 run reproduces the reference
source executed in FP64 (pinned by tests/test_oracle.py against
tests/golden/*.npz).  ``dtype=np.float32`` gives an FP32 run with the
reference's f32 constant handling (Taichi casts the Python-float ``ti.static``
constants to f32).
"""
import numpy as np

SPONGE_A = 0.0053  # forward_modeling.py:240, backward_modeling.py:243
FINITE_LIMIT = 1e30  # forward_modeling.py:482-487


def _c(x, dtype):
    return dtype(x) if dtype is np.float32 else float(x)


def sponge(nx, nz, fw, dtype=np.float64, a=SPONGE_A):
    """Cerjan sponge coefficients, forward_modeling.py:203-241.

    The reference's four loops run in order (all-ones, left, right, bottom),
    later loops overwriting earlier ones; this keeps the same order."""
    a = _c(a, dtype)
    a_sq = a * a
    c = np.ones((nx, nz), dtype)
    i = np.arange(fw)[:, None]
    j = np.arange(nz)[None, :]
    diff = (fw - np.arange(fw)).astype(dtype)
    prof = np.exp((-a_sq * diff) * diff).astype(dtype)  # -a_sq*diff*diff, left to right
    mask_lr = j < nz - i - 1
    ii, jj = np.nonzero(np.broadcast_to(mask_lr, (fw, nz)))
    keep = ii < nx
    c[ii[keep], jj[keep]] = prof[ii[keep]]  # left   (fm:214-219)
    iir = nx - ii - 1
    keep = (iir >= 0) & (iir < nx)
    c[iir[keep], jj[keep]] = prof[ii[keep]]  # right  (fm:221-227)
    i2 = np.arange(nx)[:, None]
    j2 = np.arange(fw)[None, :]
    mask_b = (i2 >= j2) & (i2 < nx - j2)
    bi, bj = np.nonzero(mask_b)
    jjb = nz - bj - 1
    keep = (jjb >= 0) & (jjb < nz)
    c[bi[keep], jjb[keep]] = prof[bj[keep]]  # bottom (fm:229-235)
    return c


def derived_material(mu, lam, rho, dtype=np.float64):
    """Averaged and inverted material, forward_modeling.py:243-307.

    Harmonic shear averages and arithmetic density averages are computed on
    the interior only (edges stay 0); the inverses cover the full grid, so
    ``inv_rho_u``/``inv_rho_w`` are +inf on the edge cells."""
    mu = np.asarray(mu, dtype)
    lam = np.asarray(lam, dtype)
    rho = np.asarray(rho, dtype)
    nx, nz = mu.shape
    I = (slice(1, nx - 1), slice(1, nz - 1))
    Ip = (slice(2, nx), slice(1, nz - 1))
    Jp = (slice(1, nx - 1), slice(2, nz))
    IJp = (slice(2, nx), slice(2, nz))
    two, four, half, one = _c(2.0, dtype), _c(4.0, dtype), _c(0.5, dtype), _c(1.0, dtype)
    out = {k: np.zeros((nx, nz), dtype) for k in ("myx", "myz", "mxz", "rho_u", "rho_w")}
    with np.errstate(all="ignore"):
        a, b, c, d = mu[I], mu[Ip], mu[Jp], mu[IJp]
        out["myx"][I] = two * a * b / (a + b)
        out["myz"][I] = two * a * c / (a + c)
        product = a * b * c * d
        s = b * c * d + a * c * d + a * b * d + a * b * c
        out["mxz"][I] = four * product / s
        out["rho_u"][I] = half * (rho[I] + rho[Ip])
        out["rho_w"][I] = half * (rho[I] + rho[Jp])
        out["inv_rho"] = one / rho
        out["inv_rho_u"] = one / out["rho_u"]
        out["inv_rho_w"] = one / out["rho_w"]
    out["mu"], out["lam"], out["rho"] = mu, lam, rho
    return out


class _State:
    def __init__(self, nx, nz, dtype):
        z = lambda: np.zeros((nx, nz), dtype)  # noqa: E731
        self.u, self.v, self.w = z(), z(), z()
        self.sxx, self.sxz, self.szz, self.syx, self.syz = z(), z(), z(), z(), z()

    def fields(self):
        return (self.u, self.v, self.w, self.sxx, self.sxz, self.szz, self.syx, self.syz)


class Propagator:
    """One propagation phase on one grid: state, material, sponge, step kernels."""

    def __init__(self, mu, lam, rho, dx, dz, fs, fw, surface=None, dtype=np.float64, setup_f64=False):
        self.dtype = dtype
        if setup_f64:
            # one-time set-up evaluated in FP64 and rounded once to ``dtype``
            # (the f32 4-point harmonic mean of fm:271 overflows for mu > ~4.3e9)
            m64 = derived_material(np.asarray(mu, np.float32), np.asarray(lam, np.float32),
                                   np.asarray(rho, np.float32), np.float64)
            self.m = {k: v.astype(dtype) for k, v in m64.items()}
            self.nx, self.nz = self.m["mu"].shape
            self.absorb = sponge(self.nx, self.nz, fw, np.float64).astype(dtype)
        else:
            self.m = derived_material(mu, lam, rho, dtype)
            self.nx, self.nz = self.m["mu"].shape
            self.absorb = sponge(self.nx, self.nz, fw, dtype)
        self.surface = None if surface is None else np.asarray(surface, dtype)
        dt = 1.0 / float(fs)  # forward_modeling.py:135
        self.dt = _c(dt, dtype)
        self.inv_dx = _c(1.0 / float(dx), dtype)
        self.inv_dz = _c(1.0 / float(dz), dtype)
        self.src_factor = _c(dt * float(dx) * float(dz), dtype)  # forward_modeling.py:430
        self.s = _State(self.nx, self.nz, dtype)
        nx, nz = self.nx, self.nz
        self.I = (slice(1, nx - 1), slice(1, nz - 1))
        self.Im = (slice(0, nx - 2), slice(1, nz - 1))
        self.Ip = (slice(2, nx), slice(1, nz - 1))
        self.Jm = (slice(1, nx - 1), slice(0, nz - 2))
        self.Jp = (slice(1, nx - 1), slice(2, nz))

    # S0 -- forward_modeling.py:404-419 / backward_modeling.py:400-415
    def surface_step(self):
        s = self.s
        if self.surface is not None:
            for f in (s.syz, s.sxz, s.szz):
                f *= self.surface
        else:
            for f in (s.syz, s.sxz, s.szz):
                f[:, 0] = 0

    # S1 forward -- forward_modeling.py:309-347
    def velocity_fwd(self):
        s, m, I, Im, Jm = self.s, self.m, self.I, self.Im, self.Jm
        dt, idx, idz = self.dt, self.inv_dx, self.inv_dz
        sxx_x = (s.sxx[I] - s.sxx[Im]) * idx
        szz_z = (s.szz[I] - s.szz[Jm]) * idz
        sxz_x = (s.sxz[I] - s.sxz[Im]) * idx
        sxz_z = (s.sxz[I] - s.sxz[Jm]) * idz
        s.u[I] += (sxx_x + sxz_z) * dt * m["inv_rho_u"][I]
        s.w[I] += (sxz_x + szz_z) * dt * m["inv_rho_w"][I]
        syx_x = (s.syx[I] - s.syx[Im]) * idx
        syz_z = (s.syz[I] - s.syz[Jm]) * idz
        s.v[I] += (syx_x + syz_z) * dt * m["inv_rho"][I]

    # S3 forward -- forward_modeling.py:349-384
    def stress_fwd(self):
        s, m, I, Ip, Jp = self.s, self.m, self.I, self.Ip, self.Jp
        dt, idx, idz = self.dt, self.inv_dx, self.inv_dz
        two = _c(2.0, self.dtype)
        u_x = (s.u[Ip] - s.u[I]) * idx
        u_z = (s.u[Jp] - s.u[I]) * idz
        w_x = (s.w[Ip] - s.w[I]) * idx
        w_z = (s.w[Jp] - s.w[I]) * idz
        div = u_x + w_z
        s.sxx[I] += dt * (m["lam"][I] * div + two * m["mu"][I] * u_x)
        s.szz[I] += dt * (m["lam"][I] * div + two * m["mu"][I] * w_z)
        s.sxz[I] += dt * m["mxz"][I] * (u_z + w_x)
        v_x = (s.v[Ip] - s.v[I]) * idx
        v_z = (s.v[Jp] - s.v[I]) * idz
        s.syx[I] += dt * m["myx"][I] * v_x
        s.syz[I] += dt * m["myz"][I] * v_z

    # S1 backward -- backward_modeling.py:312-345
    def velocity_bwd(self):
        s, m, I, Ip, Jp = self.s, self.m, self.I, self.Ip, self.Jp
        dt, idx, idz = self.dt, self.inv_dx, self.inv_dz
        sxx_x = (s.sxx[Ip] - s.sxx[I]) * idx
        szz_z = (s.szz[Jp] - s.szz[I]) * idz
        sxz_x = (s.sxz[Ip] - s.sxz[I]) * idx
        sxz_z = (s.sxz[Jp] - s.sxz[I]) * idz
        s.u[I] += -(sxx_x + sxz_z) * dt * m["inv_rho_u"][I]
        s.w[I] += -(sxz_x + szz_z) * dt * m["inv_rho_w"][I]
        syx_x = (s.syx[Ip] - s.syx[I]) * idx
        syz_z = (s.syz[Jp] - s.syz[I]) * idz
        s.v[I] += -(syx_x + syz_z) * dt * m["inv_rho"][I]

    # S3 backward -- backward_modeling.py:347-380
    def stress_bwd(self):
        s, m, I, Im, Jm = self.s, self.m, self.I, self.Im, self.Jm
        dt, idx, idz = self.dt, self.inv_dx, self.inv_dz
        two = _c(2.0, self.dtype)
        u_x = (s.u[I] - s.u[Im]) * idx
        u_z = (s.u[I] - s.u[Jm]) * idz
        w_x = (s.w[I] - s.w[Im]) * idx
        w_z = (s.w[I] - s.w[Jm]) * idz
        div = u_x + w_z
        s.sxx[I] += -dt * (m["lam"][I] * div + two * m["mu"][I] * u_x)
        s.szz[I] += -dt * (m["lam"][I] * div + two * m["mu"][I] * w_z)
        s.sxz[I] += -dt * m["mxz"][I] * (u_z + w_x)
        v_x = (s.v[I] - s.v[Im]) * idx
        v_z = (s.v[I] - s.v[Jm]) * idz
        s.syx[I] += -dt * m["myx"][I] * v_x
        s.syz[I] += -dt * m["myz"][I] * v_z

    # S4 -- forward_modeling.py:386-402
    def absorb_step(self):
        for f in self.s.fields():
            f *= self.absorb

    # S2 forward -- forward_modeling.py:421-443 (sources accumulate in order)
    def add_sources(self, src, wu, wv, ww, it):
        s, m, f = self.s, self.m, self.src_factor
        for k in range(len(src)):
            i, j = int(src[k, 0]), int(src[k, 1])
            with np.errstate(all="ignore"):
                s.u[i, j] += wu[k, it] * f * m["inv_rho_u"][i, j]
                s.v[i, j] += wv[k, it] * f * m["inv_rho"][i, j]
                s.w[i, j] += ww[k, it] * f * m["inv_rho_w"][i, j]

    # S2 backward -- backward_modeling.py:452-460
    def add_observed(self, rec, ou, ov, ow, t):
        s = self.s
        for k in range(len(rec)):
            i, j = int(rec[k, 0]), int(rec[k, 1])
            s.u[i, j] += ou[k, t]
            s.v[i, j] += ov[k, t]
            s.w[i, j] += ow[k, t]

    # forward_modeling.py:455-488 (codes 1-3) / backward_modeling.py:417-450 (4-6)
    def check_finite(self, base):
        lim = _c(FINITE_LIMIT, self.dtype)
        code = 0
        for k, f in enumerate((self.s.u, self.s.v, self.s.w)):
            with np.errstate(all="ignore"):
                bad = np.isnan(f) | (np.abs(f) > lim)
            if bad.any():
                code = base + k
        return code


def forward(mu, lam, rho, dx, dz, nt, fs, fw, src, wu, wv, ww, rec, isnap=10,
            surface=None, save=False, check_interval=100, dtype=np.float64,
            return_state=False, setup_f64=False, display_callback=None):
    """ForwardModeling.run, forward_modeling.py:504-575.

    Returns dict(flag, seis (3, nrec, nt), snaps (3, nx, nz, nsnap) or None,
    isnaps, num_snaps).  A non-zero flag returns at the failing check step,
    like the reference (the seismogram is filled up to that step).
    ``check_interval=0`` disables the finite check (used to compare with the
    Taichi-stub golden runs, whose check cannot fire).  ``setup_f64`` evaluates
    the one-time material set-up in FP64 (see Propagator).
    ``display_callback(u, v, w, it)`` gets copies of the wavefield at every
    it % isnap == 0, before that step's finite check (forward_modeling.py:553-559)."""
    p = Propagator(mu, lam, rho, dx, dz, fs, fw, surface, dtype, setup_f64)
    src = np.asarray(src).reshape(-1, 2)
    rec = np.asarray(rec).reshape(-1, 2)
    wu, wv, ww = (np.asarray(x, dtype).reshape(len(src), nt) for x in (wu, wv, ww))  # nt: also for no source
    nrec = len(rec)
    seis = np.zeros((3, nrec, nt), dtype)
    snaps = isnaps = None
    num_snaps = 0
    if save:
        num_snaps = nt // isnap
        snaps = np.zeros((3, p.nx, p.nz, num_snaps), dtype)
        isnaps = np.zeros(num_snaps, np.int32)
    ri, rj = rec[:, 0], rec[:, 1]
    flag = 0
    for it in range(nt):
        p.surface_step()
        p.velocity_fwd()
        p.add_sources(src, wu, wv, ww, it)
        p.stress_fwd()
        p.absorb_step()
        seis[0, :, it] = p.s.u[ri, rj]
        seis[1, :, it] = p.s.v[ri, rj]
        seis[2, :, it] = p.s.w[ri, rj]
        if display_callback is not None and it % isnap == 0:
            display_callback(p.s.u.copy(), p.s.v.copy(), p.s.w.copy(), it)
        if check_interval and it % check_interval == 0:
            flag = p.check_finite(1)
            if flag:
                break
        if save and it % isnap == 0 and it != 0:
            k = it // isnap - 1
            snaps[0, :, :, k] = p.s.u
            snaps[1, :, :, k] = p.s.v
            snaps[2, :, :, k] = p.s.w
            isnaps[k] = it
    out = dict(flag=flag, seis=seis, snaps=snaps, isnaps=isnaps, num_snaps=num_snaps)
    if return_state:
        out["state"] = p.s
        out["absorb"] = p.absorb
        out["material"] = p.m
    return out


def backward(mu, lam, rho, dx, dz, nt, fs, fw, rec, ou, ov, ow, snaps, isnaps, num_snaps,
             isnap, surface=None, check_interval=100, dtype=np.float64, return_state=False,
             setup_f64=False, kahan=False, display_callback=None):
    """BackwardModeling.run_calc, backward_modeling.py:498-579.

    ``snaps`` is (3, nx, nz, nsnap) like the reference's snapshot fields.
    ``kahan`` accumulates the image with Kahan compensation (sum, comp) and
    returns sum - comp evaluated in FP64 then rounded to ``dtype``.
    ``display_callback(u, v, w, t)`` gets copies of the backward wavefield
    after every imaging step (backward_modeling.py:565-569).
    Returns dict(flag, img (3, nx, nz))."""
    p = Propagator(mu, lam, rho, dx, dz, fs, fw, surface, dtype, setup_f64)
    comp = np.zeros((3, p.nx, p.nz), dtype)
    rec = np.asarray(rec).reshape(-1, 2)
    ou, ov, ow = (np.asarray(x, dtype) for x in (ou, ov, ow))
    img = np.zeros((3, p.nx, p.nz), dtype)
    flag = 0
    for it in range(nt):
        p.surface_step()
        p.velocity_bwd()
        t = (nt - 1) - it
        p.add_observed(rec, ou, ov, ow, t)
        p.stress_bwd()
        p.absorb_step()
        if t > 0 and t % isnap == 0:
            k = t // isnap - 1
            if 0 <= k < num_snaps and int(isnaps[k]) == t:
                for c, f in enumerate((p.s.u, p.s.v, p.s.w)):
                    prod = snaps[c, :, :, k] * f
                    if kahan:
                        y = prod - comp[c]
                        tot = img[c] + y
                        comp[c] = (tot - img[c]) - y
                        img[c] = tot
                    else:
                        img[c] += prod
                if display_callback is not None:
                    display_callback(p.s.u.copy(), p.s.v.copy(), p.s.w.copy(), t)
        if check_interval and it % check_interval == 0:
            flag = p.check_finite(4)
            if flag:
                break
    if kahan:
        img = (img.astype(np.float64) - comp.astype(np.float64)).astype(dtype)
    out = dict(flag=flag, img=img)
    if return_state:
        out["state"] = p.s
    return out


# ---------------------------------------------------------------- rtm.py helpers

def setup_modeling_conditions(receiver_loc, fs, estimated_v, cfl, absorbing_frame, rho0, poisson):
    """rtm.py:654-666 (homogeneous square model)."""
    dx = estimated_v / fs / cfl
    dz = dx
    nx = int((np.max(receiver_loc) - np.min(receiver_loc)) / dx)
    nx += 4 * absorbing_frame
    nz = nx
    rho = rho0 * np.ones((nx, nz), dtype=np.float32)
    vs = estimated_v * np.ones((nx, nz), dtype=np.float32)
    vp = (np.sqrt((2 * poisson + 1) / (1 - 2 * poisson)) * vs).astype(np.float32)
    return dx, dz, nx, nz, rho, vs, vp


def estimate_velocity(array, receiver_loc, source_loc, fs, vmin, vmax, vstep=10):
    """rtm.py:603-652 (geometric velocity scan, product stack)."""
    M, L = array.shape
    r = (vmax / vmin) ** (1 / (vstep - 1))
    v_array = vmin * r ** np.arange(vstep)
    sum_max = 0
    v_est = vmin
    for v in v_array:
        abs_d = np.abs(receiver_loc - source_loc)
        ts = np.round(fs * abs_d / v).astype(np.int32)
        ts = ts - np.min(ts)
        L_t = L - np.max(ts)
        if L_t <= 0:
            continue
        idx = ts[:, None] + np.arange(L_t)
        shifted = array[np.arange(M)[:, None], idx]
        sum_v = np.abs(np.sum(np.prod(shifted, axis=0)))
        if sum_v > sum_max:
            sum_max = sum_v
            v_est = v
    return float(v_est)


def imaging_slots(nt, isnap, isnaps, num_snaps):
    """Snapshot slots the cross-correlation uses, in backward order: slot
    k = t // isnap - 1 at every reversed time t > 0 with t % isnap == 0 and
    isnaps[k] == t (backward_modeling.py:556-564)."""
    out = []
    for it in range(nt):
        t = (nt - 1) - it
        if t > 0 and t % isnap == 0:
            k = t // isnap - 1
            if 0 <= k < num_snaps and int(isnaps[k]) == t:
                out.append(k)
    return out


def source_normalized(img, snaps, slots, eps):
    """Source-normalised zero-lag cross-correlation.  No reference
    counterpart: the reference accepts an imaging ``method`` and ignores it
    (backward_modeling.py:505).  The definition restated here: per component c,
    I_c = sum over the used snapshot slots of snapshot_c^2 (FP64) and
    image_c = xcorr_c / (I_c + eps * max I_c), 0 where that divisor is 0.
    ``img`` is (3, nx, nz), ``snaps`` (3, nx, nz, nsnap)."""
    out = np.zeros(np.shape(img), np.float64)
    for c in range(3):
        ill = np.zeros(np.shape(img)[1:], np.float64)
        for k in slots:
            s = np.asarray(snaps[c, :, :, k], np.float64)
            ill += s * s
        d = ill + eps * ill.max()
        out[c] = np.where(d > 0, np.asarray(img[c], np.float64) / np.where(d > 0, d, 1.0), 0.0)
    return out
