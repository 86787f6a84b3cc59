"""rtm_forward_noalloc: the forward entry point that allocates no device memory.

It is meant for callers that cannot call cudaMalloc while running -- for
example a plugin inside a host processing system that owns every byte of
device memory and gives the plugin only a stream and its buffers.  These
tests call it through the C ABI and check it against rtm_forward, the
plan-based entry point, run with the same launch shape (vec 2, 16 rows, 4
warps, one step per launch): the seismograms and the status must be equal bit
for bit, on two calls in a row (different inputs each time, so state left in
the shared scratch by the first call must not leak into the second) and for
P-SV only, SH only, no receivers and no sponge.  A call after the set-up must
leave the device's free memory unchanged.  The file is named to be collected
last."""
import ctypes

import numpy as np
import pytest
import torch

from taichirtm_b200 import _lib
from taichirtm_b200.plan import BOTH, PSV, SH, Plan, ShotGeometry

pytestmark = pytest.mark.gpu

SHAPE = dict(vec=2, rows=16, warps=4, prefetch=0, tsteps=1)  # the entry point's launch shape


def _bind():
    L = _lib.lib()
    f = L.rtm_forward_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.RtmGrid), ctypes.c_int, _lib.I32P, ctypes.c_int, _lib.I32P,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int, _lib.I32P, ctypes.c_void_p]
    L.rtm_noalloc_prepare.restype = ctypes.c_int
    L.rtm_noalloc_prepare.argtypes = []
    L.rtm_noalloc_scratch_bytes.restype = ctypes.c_size_t
    L.rtm_noalloc_required_bytes.restype = ctypes.c_size_t
    L.rtm_noalloc_required_bytes.argtypes = [ctypes.POINTER(_lib.RtmGrid), ctypes.c_int, ctypes.c_int]
    L.rtm_noalloc_last_error.restype = ctypes.c_char_p
    return L


def _model(nx, nz, seed):
    rng = np.random.default_rng(seed)
    vp = 2000.0 + 800.0 * rng.random((nx, nz))
    vs, rho = vp / 1.73, 310.0 * vp ** 0.25
    mu = (rho * vs ** 2).astype(np.float32)
    lam = (rho * vp ** 2 - 2 * rho * vs ** 2).astype(np.float32)
    return mu, lam, rho.astype(np.float32)


def _case(seed, nx=90, nz=70, nt=260, modes=BOTH, fw=12, nrec=None):
    mu, lam, rho = _model(nx, nz, seed)
    t = np.arange(nt) / 2000.0
    a = (np.pi * 50.0 * (t - 0.02)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.array([[nx // 2 + seed, 3], [nx // 3, 9]], np.int32)
    wav = np.stack([np.stack([0.5 * w, 0.1 * w]), np.stack([0.3 * w, 0.2 * w]), np.stack([w, 0.6 * w])])
    if not modes & PSV:
        wav[[0, 2]] = 0.0
    if not modes & SH:
        wav[1] = 0.0
    cols = np.arange(seed % 3, nx, 2)
    rec = np.stack([cols, np.ones(len(cols), int)], 1).astype(np.int32)
    if nrec is not None:
        rec = rec[:nrec]
    return dict(mu=mu, lam=lam, rho=rho, src=src, rec=rec, wav=wav.astype(np.float32), nx=nx, nz=nz, nt=nt,
                modes=modes, fw=fw)


def _grid(c):
    return _lib.RtmGrid(c["nx"], c["nz"], 5.0, 5.0, 2000.0, c["nt"], c["fw"], c["modes"])


def _existing(c):
    p = Plan(c["nx"], c["nz"], 5.0, 5.0, c["nt"], 2000.0, c["fw"], c["modes"],
             [ShotGeometry(0, c["nx"], c["src"], c["rec"])], tune=SHAPE)
    p.set_model(c["mu"], c["lam"], c["rho"])
    flags, seis, _, _ = p.forward(torch.as_tensor(c["wav"]), check_interval=100)
    out = seis.cpu().numpy()
    p.close()
    return int(flags[0]), out


class _Call:
    """Device inputs and outputs of one call, allocated up front."""

    def __init__(self, L, c):
        dev = torch.device("cuda")
        self.L, self.c = L, c
        self.mu, self.lam, self.rho = (torch.as_tensor(c[k]).to(dev).contiguous() for k in ("mu", "lam", "rho"))
        self.wav = torch.as_tensor(c["wav"]).to(dev).contiguous()
        self.seis = torch.full((3, len(c["rec"]), c["nt"]), float("nan"), device=dev)
        self.flag = np.zeros(1, np.int32)
        self.g = _grid(c)

    def __call__(self):
        c = self.c
        rc = self.L.rtm_forward_noalloc(ctypes.byref(self.g), len(c["src"]), c["src"].ctypes.data_as(_lib.I32P),
                                        len(c["rec"]), c["rec"].ctypes.data_as(_lib.I32P), self.mu.data_ptr(),
                                        self.lam.data_ptr(), self.rho.data_ptr(), self.wav.data_ptr(),
                                        self.seis.data_ptr(), 100, self.flag.ctypes.data_as(_lib.I32P),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, self.L.rtm_noalloc_last_error()
        return int(self.flag[0])


def _check_equal(L, c):
    need = L.rtm_noalloc_required_bytes(ctypes.byref(_grid(c)), len(c["src"]), len(c["rec"]))
    assert 0 < need <= L.rtm_noalloc_scratch_bytes()
    f_ref, ref = _existing(c)
    call = _Call(L, c)
    f_new = call()
    new = call.seis.cpu().numpy()
    assert f_ref == 0 and f_new == 0
    assert new.shape == ref.shape
    assert np.array_equal(new, ref)


def test_noalloc_equals_rtm_forward_on_two_calls_in_a_row():
    L = _bind()
    assert L.rtm_noalloc_prepare() == 0, L.rtm_noalloc_last_error()
    for seed in (1, 2):
        _check_equal(L, _case(seed))


@pytest.mark.parametrize("kind", ["psv_only", "sh_only", "no_receivers", "no_sponge"])
def test_noalloc_equals_rtm_forward_variants(kind):
    L = _bind()
    c = {"psv_only": lambda: _case(3, modes=PSV), "sh_only": lambda: _case(4, modes=SH),
         "no_receivers": lambda: _case(5, nrec=0), "no_sponge": lambda: _case(6, fw=0)}[kind]()
    _check_equal(L, c)


def test_noalloc_call_after_setup_leaves_device_memory_unchanged():
    L = _bind()
    assert L.rtm_noalloc_prepare() == 0, L.rtm_noalloc_last_error()
    c = _case(7)
    call = _Call(L, c)
    assert call() == 0  # first call on this device (after the set-up)
    ref = call.seis.cpu().numpy()
    for modes in (PSV, SH, BOTH):  # every kernel instantiation the entry point launches
        _Call(L, _case(8, modes=modes))()
    call2 = _Call(L, c)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call2() == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.array_equal(call2.seis.cpu().numpy(), ref)


def test_noalloc_rejects_sizes_above_its_limit():
    L = _bind()
    c = _case(1)
    g = _lib.RtmGrid(3000, 3000, 5.0, 5.0, 2000.0, 100, 12, BOTH)
    assert L.rtm_noalloc_required_bytes(ctypes.byref(g), 2, len(c["rec"])) > L.rtm_noalloc_scratch_bytes()
    flag = np.zeros(1, np.int32)
    rc = L.rtm_forward_noalloc(ctypes.byref(g), len(c["src"]), c["src"].ctypes.data_as(_lib.I32P),
                               len(c["rec"]), c["rec"].ctypes.data_as(_lib.I32P), 1, 1, 1, 1, 1, 100,
                               flag.ctypes.data_as(_lib.I32P), None)
    assert rc == -5
    assert b"limit" in L.rtm_noalloc_last_error()
