"""The ctypes binding a TaichiRTM maintainer would add to use librtm_b200.

TaichiRTM is pure Python (its boundary is ``src/__init__.py:24-55``), so its
binding to this library is ``ctypes``.  ``run_forward`` keeps the arguments of
``ForwardModeling`` (src/forward_modeling.py:126-153) and replaces its time
loop (src/forward_modeling.py:504-575) with one ``rtm_forward`` call.  The
fields are device arrays (torch or cupy); their ``data_ptr()`` values are the
device pointers.  The package's own binding (``_lib.py``, ``plan.py``) is this
stub in full: argument types for every symbol, snapshot buffers and error
translation.
"""
import ctypes

import numpy as np

LIBRARY = "librtm_b200.so"


class RtmGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_double),
                ("dz", ctypes.c_double), ("fs", ctypes.c_double), ("nt", ctypes.c_int),
                ("absorbing_frame", ctypes.c_int), ("modes", ctypes.c_int)]


class RtmShot(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int), ("nx", ctypes.c_int), ("nsrc", ctypes.c_int),
                ("src_ij", ctypes.POINTER(ctypes.c_int32)), ("nrec", ctypes.c_int),
                ("rec_ij", ctypes.POINTER(ctypes.c_int32))]


def load(path=LIBRARY):
    lib = ctypes.CDLL(path)
    lib.rtm_last_error.restype = ctypes.c_char_p
    return lib


def run_forward(lib, nx, nz, dx, dz, nt, fs, fw, mu, lam, rho, src_ij, rec_ij, wavelets, seis, stream=0):
    """mu/lam/rho (nx,nz), wavelets (3,nsrc,nt), seis (3,nrec,nt): device arrays.
    Returns 0, or 1/2/3 like ForwardModeling.run."""
    g = RtmGrid(nx, nz, dx, dz, fs, nt, fw, 3)  # P-SV + SH, as the reference runs
    src = np.ascontiguousarray(src_ij, np.int32)
    rec = np.ascontiguousarray(rec_ij, np.int32)
    shot = RtmShot(0, nx, len(src), src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                   len(rec), rec.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    plan = ctypes.c_void_p()
    if lib.rtm_plan_create(ctypes.byref(g), 1, ctypes.byref(shot), None, ctypes.byref(plan)) != 0:
        raise RuntimeError(lib.rtm_last_error().decode())
    try:
        if lib.rtm_plan_set_model(plan, ctypes.c_void_p(mu.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                  ctypes.c_void_p(rho.data_ptr()), None, ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(lib.rtm_last_error().decode())
        flag = np.zeros(1, np.int32)
        rc = lib.rtm_forward(plan, ctypes.c_void_p(wavelets.data_ptr()), ctypes.c_void_p(seis.data_ptr()),
                             0, 10, None, None, None, None, 100,
                             flag.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(lib.rtm_last_error().decode())
        return int(flag[0])
    finally:
        lib.rtm_plan_destroy(plan)
