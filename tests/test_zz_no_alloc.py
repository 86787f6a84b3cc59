"""rtm_forward_noalloc: the forward entry point that allocates no device memory.

It is meant for callers that cannot call cudaMalloc while running -- for
example a plugin inside a host processing system that owns every byte of
device memory and gives the plugin only a stream and its buffers.  This test
calls it through the C ABI twice in a row (different inputs each time, so
state left in the shared scratch by the first call must not leak into the
second) and checks each result against rtm_forward, the plan-based entry
point, within the seismogram tolerance of the parity tests (relative L2
1e-5).  The file is named to be collected last."""
import ctypes

import numpy as np
import pytest
import torch

from taichirtm_b200 import _lib
from taichirtm_b200.plan import BOTH, Plan, ShotGeometry
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5


def _bind():
    L = _lib.lib()
    f = L.rtm_forward_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.RtmGrid), ctypes.c_int, _lib.I32P, ctypes.c_int, _lib.I32P,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int, _lib.I32P, ctypes.c_void_p]
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


def _case(seed, nx=90, nz=70, nt=260):
    mu, lam, rho = _model(nx, nz, seed)
    t = np.arange(nt) / 2000.0
    a = (np.pi * 50.0 * (t - 0.02)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.array([[nx // 2 + seed, 3], [nx // 3, 9]], np.int32)
    wav = np.stack([np.stack([0.5 * w, 0.1 * w]), np.stack([0.3 * w, 0.2 * w]), np.stack([w, 0.6 * w])])
    rec = np.stack([np.arange(seed % 3, nx, 2), np.ones(len(range(seed % 3, nx, 2)), int)], 1).astype(np.int32)
    return dict(mu=mu, lam=lam, rho=rho, src=src, rec=rec, wav=wav.astype(np.float32), nx=nx, nz=nz, nt=nt)


def _grid(c):
    return _lib.RtmGrid(c["nx"], c["nz"], 5.0, 5.0, 2000.0, c["nt"], 12, BOTH)


def _existing(c):
    p = Plan(c["nx"], c["nz"], 5.0, 5.0, c["nt"], 2000.0, 12, BOTH, [ShotGeometry(0, c["nx"], c["src"], c["rec"])])
    p.set_model(c["mu"], c["lam"], c["rho"])
    flags, seis, _, _ = p.forward(torch.as_tensor(c["wav"]), check_interval=100)
    out = seis.cpu().numpy()
    p.close()
    return int(flags[0]), out


def _noalloc(L, c):
    dev = torch.device("cuda")
    mu, lam, rho = (torch.as_tensor(c[k]).to(dev).contiguous() for k in ("mu", "lam", "rho"))
    wav = torch.as_tensor(c["wav"]).to(dev).contiguous()
    seis = torch.full((3, len(c["rec"]), c["nt"]), float("nan"), device=dev)
    flag = np.zeros(1, np.int32)
    g = _grid(c)
    rc = L.rtm_forward_noalloc(ctypes.byref(g), len(c["src"]), c["src"].ctypes.data_as(_lib.I32P),
                               len(c["rec"]), c["rec"].ctypes.data_as(_lib.I32P), mu.data_ptr(),
                               lam.data_ptr(), rho.data_ptr(), wav.data_ptr(), seis.data_ptr(), 100,
                               flag.ctypes.data_as(_lib.I32P),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.rtm_noalloc_last_error()
    return int(flag[0]), seis.cpu().numpy()


def test_noalloc_matches_rtm_forward_on_two_calls_in_a_row():
    L = _bind()
    for seed in (1, 2):
        c = _case(seed)
        need = L.rtm_noalloc_required_bytes(ctypes.byref(_grid(c)), len(c["src"]), len(c["rec"]))
        assert 0 < need <= L.rtm_noalloc_scratch_bytes()
        f_ref, ref = _existing(c)
        f_new, new = _noalloc(L, c)
        assert f_ref == 0 and f_new == 0
        assert np.isfinite(new).all()
        e = rel_l2(new, ref)
        assert e <= SEIS_TOL, (seed, e)


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
