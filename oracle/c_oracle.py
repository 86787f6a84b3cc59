"""ctypes wrapper of the C/OpenMP restatement (oracle/rtm_oracle.c) -- TEST
INFRASTRUCTURE: the checker at sizes NumPy is slow for, and the timed CPU
baseline.  Build with ``make -C oracle`` (``__graft_entry__.build()`` does)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "librtm_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def max_threads():
    return int(lib().rtm_oracle_max_threads_f32())


def _comps_mask(snap_comps):
    return sum(1 << c for c in sorted(set(snap_comps)))


def forward(mu, lam, rho, dx, dz, nt, fs, fw, src, wu, wv, ww, rec, isnap=10, surface=None,
            save=False, check_interval=100, dtype=np.float32, modes=3, nthreads=0, nt_run=0,
            setup_f64=True, snap_comps=(0, 1, 2)):
    """ForwardModeling.run restated in C.  ``setup_f64`` evaluates the one-time
    material averages in double (see rtm_oracle.c: the reference's f32 4-point
    harmonic mean overflows for mu > ~4.3e9 Pa).  ``snap_comps``: the
    components (0 u, 1 v, 2 w) whose snapshots are kept, in that order (the
    others image as zero in ``backward``).  Returns dict(flag, seis (3, nrec,
    nt), snaps (len(snap_comps), nsnap, nx, nz) or None, isnaps, num_snaps,
    snap_comps)."""
    snap_comps = tuple(sorted(set(snap_comps)))
    sfx = "f32" if dtype == np.float32 else "f64"
    mu, lam, rho = (np.ascontiguousarray(x, dtype) for x in (mu, lam, rho))
    nx, nz = mu.shape
    src = np.ascontiguousarray(np.asarray(src).reshape(-1, 2), np.int32)
    rec = np.ascontiguousarray(np.asarray(rec).reshape(-1, 2), np.int32)
    wu, wv, ww = (np.ascontiguousarray(np.asarray(x).reshape(len(src), nt), dtype) for x in (wu, wv, ww))
    sm = None if surface is None else np.ascontiguousarray(surface, dtype)
    seis = np.zeros((3, len(rec), nt), dtype)
    num_snaps = nt // isnap if save else 0
    snaps = np.zeros((len(snap_comps), num_snaps, nx, nz), dtype) if save else None
    isnaps = np.zeros(max(num_snaps, 1), np.int32)
    f = getattr(lib(), "rtm_oracle_forward_" + sfx)
    flag = f(ctypes.c_int(nx), ctypes.c_int(nz), ctypes.c_double(dx), ctypes.c_double(dz),
             ctypes.c_int(nt), ctypes.c_double(fs), ctypes.c_int(fw), _p(mu), _p(lam), _p(rho),
             _p(sm), ctypes.c_int(len(src)), _p(src), _p(wu), _p(wv), _p(ww),
             ctypes.c_int(len(rec)), _p(rec), _p(seis), ctypes.c_int(isnap), ctypes.c_int(int(save)),
             _p(snaps), _p(isnaps), ctypes.c_int(check_interval), ctypes.c_int(modes),
             ctypes.c_int(nthreads), ctypes.c_int(nt_run), ctypes.c_int(int(setup_f64)),
             ctypes.c_int(_comps_mask(snap_comps)))
    return dict(flag=int(flag), seis=seis, snaps=snaps, isnaps=isnaps[:num_snaps], num_snaps=num_snaps,
                snap_comps=snap_comps)


def backward(mu, lam, rho, dx, dz, nt, fs, fw, rec, obs, snaps, isnaps, num_snaps, isnap,
             surface=None, check_interval=100, dtype=np.float32, modes=3, nthreads=0, nt_run=0,
             setup_f64=True, snap_comps=(0, 1, 2)):
    """BackwardModeling.run_calc restated in C.  ``obs`` is (3, nrec, nt),
    ``snaps`` (len(snap_comps), nsnap, nx, nz) holding the components
    ``snap_comps`` (the forward's).  Returns dict(flag, img (3, nx, nz))."""
    snap_comps = tuple(sorted(set(snap_comps)))
    sfx = "f32" if dtype == np.float32 else "f64"
    mu, lam, rho = (np.ascontiguousarray(x, dtype) for x in (mu, lam, rho))
    nx, nz = mu.shape
    rec = np.ascontiguousarray(np.asarray(rec).reshape(-1, 2), np.int32)
    obs = np.ascontiguousarray(obs, dtype)
    snaps = np.ascontiguousarray(snaps, dtype)
    if snaps.shape[0] != len(snap_comps):
        raise ValueError(f"snaps holds {snaps.shape[0]} components, snap_comps names {len(snap_comps)}")
    isnaps = np.ascontiguousarray(np.asarray(isnaps).reshape(-1), np.int32)
    if isnaps.size == 0:
        isnaps = np.zeros(1, np.int32)
    sm = None if surface is None else np.ascontiguousarray(surface, dtype)
    img = np.zeros((3, nx, nz), dtype)
    f = getattr(lib(), "rtm_oracle_backward_" + sfx)
    flag = f(ctypes.c_int(nx), ctypes.c_int(nz), ctypes.c_double(dx), ctypes.c_double(dz),
             ctypes.c_int(nt), ctypes.c_double(fs), ctypes.c_int(fw), _p(mu), _p(lam), _p(rho),
             _p(sm), ctypes.c_int(len(rec)), _p(rec), _p(obs), _p(snaps), _p(isnaps),
             ctypes.c_int(num_snaps), ctypes.c_int(isnap), _p(img), ctypes.c_int(check_interval),
             ctypes.c_int(modes), ctypes.c_int(nthreads), ctypes.c_int(nt_run),
             ctypes.c_int(int(setup_f64)), ctypes.c_int(_comps_mask(snap_comps)))
    return dict(flag=int(flag), img=img)
