"""Two time steps per launch (tune tsteps=2, temporal blocking) against one
step per launch: every output must be bit-identical, because each cell's FP32
arithmetic is the same operation sequence.

Covered: P-SV, SH and both; vec 2 / 4; row tasks of 1, 2, 7, 16 rows (the
recomputed halo rows of step A at every task edge); several column strips
with sources and receivers on the strip and task boundaries; topography;
odd nt (the last launch is a single step); snapshots at odd and even steps;
backward imaging with both steps of a pair imaging (isnap 1); the finite
check (the same code at the same step); windowed batched shots; the
checkpointed forward / backward and the FWI gradient.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _model(nx, nz, seed):
    from taichirtm_b200.synthetic import gaussian_smooth
    rng = np.random.default_rng(seed)
    vp = 1800.0 + 1400.0 * np.linspace(0, 1, nz)[None, :] + 300.0 * gaussian_smooth(rng.standard_normal((nx, nz)), 3)
    vp = np.clip(vp, 1500.0, 3600.0)
    vs = vp / 1.8
    rho = 310.0 * vp ** 0.25
    mu = (rho * vs ** 2).astype(np.float32)
    lam = (rho * vp ** 2 - 2 * rho * vs ** 2).astype(np.float32)
    return mu, lam, rho.astype(np.float32)


def _ricker(nt, fs, f0, shift):
    t = np.arange(nt) / fs - shift
    a = (np.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _case(nx=157, nz=203, nt=61, fw=20, seed=3):
    # sources on strip boundaries (vec 2: 60-column strips; vec 4: 120) and
    # near task boundaries; receivers along j = 1 plus a vertical line
    src = np.array([[nx // 2, 2], [41, 59], [48, 60], [63, 119], [96, 120], [112, 61]], np.int32)
    rec = [[i, 1] for i in range(nx)] + [[70, j] for j in range(2, nz - 1, 3)] + [[16, 59], [32, 60], [33, 121]]
    rec = np.array(rec, np.int32)
    inside = lambda a: a[(a[:, 0] < nx) & (a[:, 1] < nz)]  # noqa: E731
    src, rec = inside(src), inside(rec)
    wav = np.zeros((3, len(src), nt), np.float32)
    for k in range(len(src)):
        w = _ricker(nt, 2000.0, 60.0, 0.012 + 0.001 * k)
        wav[0, k], wav[1, k], wav[2, k] = 0.4 * w, 0.7 * w, w
    return dict(nx=nx, nz=nz, nt=nt, fw=fw, dx=4.0, dz=4.0, fs=2000.0, src=src, rec=rec, wav=wav,
                model=_model(nx, nz, seed))


def _topography(nx, nz):
    sm = np.ones((nx, nz), np.float32)
    h = (4 + 3 * np.sin(np.arange(nx) / 9.0)).astype(int)
    for i in range(nx):
        sm[i, :h[i]] = 0.0
    return sm


def _run(C, modes, tune, isnap, check=7, surface=None):
    from taichirtm_b200.plan import Plan, ShotGeometry
    p = Plan(C["nx"], C["nz"], C["dx"], C["dz"], C["nt"], C["fs"], C["fw"], modes,
             [ShotGeometry(0, C["nx"], C["src"], C["rec"])], tune=tune)
    mu, lam, rho = C["model"]
    p.set_model(mu, lam, rho, surface)
    ff, seis, snaps, isn = p.forward(torch.as_tensor(C["wav"]), save=True, isnap=isnap, check_interval=check)
    obs = seis.flip(-1).contiguous() * 0.5 + seis
    fb, img, _ = p.backward(obs, snaps, isn, len(isn), isnap, check_interval=check)
    out = dict(ff=ff.copy(), fb=fb.copy(), seis=seis.cpu().numpy(), img=img.cpu().numpy(),
               snaps=[None if s is None else s.cpu().numpy() for s in snaps], launches=p.launch_count())
    p.close()
    return out


def _same(a, b):
    """Bit-identical outputs; NaN (after a failed check) compares equal to NaN."""
    assert np.array_equal(a["ff"], b["ff"]) and np.array_equal(a["fb"], b["fb"])
    assert np.array_equal(a["seis"], b["seis"], equal_nan=True)
    assert np.array_equal(a["img"], b["img"], equal_nan=True)
    for x, y in zip(a["snaps"], b["snaps"]):
        assert (x is None) == (y is None)
        if x is not None:
            assert np.array_equal(x, y, equal_nan=True)


@pytest.mark.parametrize("modes", [1, 2, 3])
@pytest.mark.parametrize("tune", [dict(vec=2, rows=7, warps=3), dict(vec=4, rows=16, warps=2),
                                  dict(vec=2, rows=1, warps=4), dict(vec=4, rows=2, warps=1),
                                  dict(vec=2, rows=5, warps=2, prefetch=3), dict(vec=4, rows=3, warps=1, prefetch=3),
                                  dict(vec=2, rows=1, warps=8, prefetch=3), dict(vec=2, rows=5, warps=1, prefetch=4),
                                  dict(vec=4, rows=3, warps=1, prefetch=4)])
def test_two_steps_per_launch_bit_identical(modes, tune):
    C = _case()
    one = _run(C, modes, dict(tune, tsteps=1), isnap=3)
    two = _run(C, modes, dict(tune, tsteps=2), isnap=3)
    assert np.abs(one["img"]).max() > 0 and np.abs(one["seis"]).max() > 0
    _same(one, two)
    assert two["launches"] < one["launches"]


@pytest.mark.parametrize("prefetch", [1, 3, 4])
@pytest.mark.parametrize("isnap", [1, 2])
def test_two_steps_imaging_every_step_and_topography(isnap, prefetch):
    C = _case(nx=90, nz=130, nt=40, fw=12, seed=5)
    sm = _topography(C["nx"], C["nz"])
    one = _run(C, 1, dict(vec=2, rows=5, warps=2, tsteps=1), isnap=isnap, check=1, surface=sm)
    two = _run(C, 1, dict(vec=2, rows=5, warps=2, tsteps=2, prefetch=prefetch), isnap=isnap, check=1, surface=sm)
    _same(one, two)
    two = _run(C, 1, dict(vec=2, rows=5, warps=2, tsteps=2, prefetch=prefetch), isnap=isnap, check=0, surface=sm)
    _same(one, two)


def test_two_steps_failure_code_at_same_step():
    """A source on an edge cell injects inf (1/rho = inf there): the check
    must report the same code as one step per launch, for check intervals
    that put checked steps at either position of a pair."""
    C = _case(nx=60, nz=70, nt=30, fw=8)
    C["src"] = np.array([[0, 30]], np.int32)
    C["wav"] = C["wav"][:, :1]
    for check in (1, 2, 3, 5):
        a = _run(C, 3, dict(vec=2, rows=4, warps=2, tsteps=1), isnap=2, check=check)
        b = _run(C, 3, dict(vec=2, rows=4, warps=2, tsteps=2), isnap=2, check=check)
        assert a["ff"][0] == 3
        _same(a, b)


def _batched(tsteps, checkpoint=None, modes=1):
    from taichirtm_b200.batch import BatchedRTM
    from taichirtm_b200.plan import ShotGeometry
    nx, nz, nt, fw = 260, 150, 57, 16
    mu, lam, rho = _model(nx, nz, 11)
    shots, wav = [], []
    for k, (x0, w) in enumerate([(0, 120), (70, 101), (139, 121), (30, 230)]):
        src = np.array([[w // 2, 2]], np.int32)
        rec = np.stack([np.arange(0, w, 2), np.ones(len(range(0, w, 2)), int)], 1).astype(np.int32)
        shots.append(ShotGeometry(x0, w, src, rec))
        wav.append(_ricker(nt, 2000.0, 50.0, 0.015))
    wv = np.zeros((3, len(shots), nt), np.float32)
    wv[2] = np.stack(wav)
    wv[0] = 0.3 * wv[2]
    b = BatchedRTM(mu, lam, rho, 4.0, 4.0, 2000.0, nt, fw, shots, modes=modes,
                   tune=dict(vec=2, rows=9, warps=2, tsteps=tsteps, prefetch=3 if tsteps == 2 else 1),
                   graphs=tsteps == 2)
    ff, seis, _, _ = b.forward(wv, check_interval=10)
    obs = seis * 0.7
    out = b.migrate(wv, obs, isnap=3, check_interval=10, checkpoint=checkpoint)
    res = (seis.cpu().numpy(), out[2].cpu().numpy(), out[0].copy(), out[1].copy())
    b.close()
    return res


@pytest.mark.parametrize("checkpoint", [None, dict(every=8, dtype="f32"), dict(every=7, dtype="f16"),
                                        dict(every=7, dtype="i16")])
def test_two_steps_batched_windows_and_checkpointed(checkpoint):
    a = _batched(1, checkpoint)
    b = _batched(2, checkpoint)
    assert np.abs(a[1]).max() > 0
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_two_steps_fwi_gradient_bit_identical():
    from taichirtm_b200.fwi import FWIProblem
    from taichirtm_b200.plan import ShotGeometry
    C = _case(nx=80, nz=64, nt=90, fw=10)
    mu, lam, rho = C["model"]
    src = C["src"][:1]
    src[0] = [40, 3]
    rec = np.stack([np.arange(10, 70, 2), np.full(30, 2)], 1).astype(np.int32)
    grads = []
    for ts in (1, 2):
        prob = FWIProblem(C["nx"], C["nz"], C["dx"], C["dz"], C["fs"], C["nt"], C["fw"],
                          [ShotGeometry(0, C["nx"], src, rec)], C["wav"][:, :1], ckpt_every=9,
                          tune=dict(vec=2, rows=8, warps=2, tsteps=ts))
        seis, ck, flags = prob.forward(lam, mu, rho)
        g = prob.adjoint(seis * 0.5, ck)
        grads.append((seis.cpu().numpy(), g[0].cpu().numpy() if isinstance(g, tuple) else g.cpu().numpy()))
    assert np.array_equal(grads[0][0], grads[1][0])
    assert np.array_equal(grads[0][1], grads[1][1])


def test_failing_check_step_is_complete_for_every_launch_shape():
    """A huge wavelet sample at step 7 overflows the check threshold; the check
    at step 10 (interval 5) fails.  The reference records step 10 in full and
    then returns (forward_modeling.py:550-566), so every warp of the failing
    launch must finish its rows: the seismograms, up to and including step
    10, are bit-identical for every launch shape (one and two steps per
    launch, different warps per CTA) and to the NumPy FP32 restatement, which
    stops at the same check; later samples stay zero."""
    from oracle import fd_oracle
    from taichirtm_b200.plan import Plan, ShotGeometry
    C = _case(nx=64, nz=70, nt=24, fw=8)
    src = np.array([[32, 6]], np.int32)  # the step-2 pulse reaches the j = 1 receivers by step 10
    wav = np.zeros((3, 1, C["nt"]), np.float32)
    wav[2, 0, 2] = 1.0
    wav[2, 0, 7] = 1e36
    mu, lam, rho = C["model"]
    kw = dict(dx=C["dx"], dz=C["dz"], nt=C["nt"], fs=C["fs"], fw=C["fw"])
    with np.errstate(over="ignore", invalid="ignore"):  # the blow-up is the point
        ref = fd_oracle.forward(mu, lam, rho, src=src, wu=wav[0, 0], wv=wav[1, 0], ww=wav[2, 0], rec=C["rec"],
                                check_interval=5, dtype=np.float32, setup_f64=True, **kw)
    assert ref["flag"] in (1, 3)
    outs = []
    for tune in (dict(vec=2, rows=4, warps=2, tsteps=1), dict(vec=2, rows=4, warps=2, tsteps=2),
                 dict(vec=1, rows=3, warps=1, prefetch=0), dict(vec=4, rows=64, warps=8, prefetch=3),
                 dict(vec=4, rows=2, warps=8, tsteps=2), dict(vec=2, rows=6, warps=2, tsteps=2, prefetch=3),
                 dict(vec=2, rows=6, warps=1, tsteps=2, prefetch=4)):
        p = Plan(C["nx"], C["nz"], C["dx"], C["dz"], C["nt"], C["fs"], C["fw"], 1,
                 [ShotGeometry(0, C["nx"], src, C["rec"])], tune=tune)
        p.set_model(mu, lam, rho)
        f, seis, _, _ = p.forward(torch.as_tensor(wav), check_interval=5)
        outs.append((int(f[0]), seis.cpu().numpy()))
        p.close()
    for code, seis in outs:
        assert code == ref["flag"]
        assert np.array_equal(seis[[0, 2]], ref["seis"][[0, 2]], equal_nan=True)
        assert np.abs(seis[:, :, 11:]).max() == 0.0
        assert np.nanmax(np.abs(seis[:, :, 10])) > 0.0
