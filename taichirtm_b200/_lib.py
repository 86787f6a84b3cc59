"""ctypes binding of librtm_b200.so (include/rtm_b200.h).

The product path has no fallback: if the library is missing or fails to load
this module raises, and every propagation call goes through it."""
import ctypes
import os

from . import build as _build

I32P = ctypes.POINTER(ctypes.c_int32)
# rtm_step_callback: int (*)(void *user, int step)
STEP_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)


class RtmGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_double),
                ("dz", ctypes.c_double), ("fs", ctypes.c_double), ("nt", ctypes.c_int),
                ("absorbing_frame", ctypes.c_int), ("modes", ctypes.c_int)]


class RtmShot(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int), ("nx", ctypes.c_int), ("nsrc", ctypes.c_int),
                ("src_ij", I32P), ("nrec", ctypes.c_int), ("rec_ij", I32P)]


class RtmTune(ctypes.Structure):
    _fields_ = [("vec", ctypes.c_int), ("rows", ctypes.c_int), ("warps", ctypes.c_int),
                ("prefetch", ctypes.c_int), ("graphs", ctypes.c_int), ("tsteps", ctypes.c_int)]


PSV, SH, BOTH = 1, 2, 3
CKPT_DTYPES = {"f32": 0, "f16": 1, "bf16": 2, "i16": 3}
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "call out of order", -4: "out of device memory",
          -5: "size above the entry point's limit", -6: "stopped by the step callback"}

_lib = None


class RtmError(RuntimeError):
    def __init__(self, code, fn):
        msg = lib().rtm_last_error().decode(errors="replace")
        super().__init__(f"{fn}: {ERRORS.get(code, code)} ({code}): {msg}")
        self.code = code


def _sig(L, name, restype, *args):
    f = getattr(L, name)
    f.restype = restype
    f.argtypes = list(args)


def lib():
    """Load librtm_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    override = os.environ.get("TAICHIRTM_B200_LIB")  # a separately built librtm_b200.so
    path = override or _build.LIB
    if not override and (not os.path.exists(path) or _build._stale(path)):
        try:
            path = _build.build()
        except Exception as e:  # no nvcc: fail loudly, there is no CPU path
            if not os.path.exists(path):
                raise RuntimeError("librtm_b200.so is missing and could not be built: %s" % e)
    L = ctypes.CDLL(path)
    vp, c_int, c_size = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    _sig(L, "rtm_version", ctypes.c_char_p)
    _sig(L, "rtm_last_error", ctypes.c_char_p)
    _sig(L, "rtm_plan_create", c_int, ctypes.POINTER(RtmGrid), c_int, ctypes.POINTER(RtmShot),
         ctypes.POINTER(RtmTune), ctypes.POINTER(vp))
    _sig(L, "rtm_plan_destroy", c_int, vp)
    _sig(L, "rtm_plan_pitch", c_int, vp)
    _sig(L, "rtm_plan_snapshot_floats", c_size, vp, c_int)
    _sig(L, "rtm_plan_launch_count", ctypes.c_longlong, vp)
    _sig(L, "rtm_plan_set_model", c_int, vp, vp, vp, vp, vp, vp)
    _sig(L, "rtm_forward", c_int, vp, vp, vp, c_int, c_int, vp, vp, vp, I32P, c_int, I32P, vp)
    _sig(L, "rtm_backward", c_int, vp, vp, vp, vp, vp, I32P, c_int, c_int, vp, vp, c_int, I32P, vp)
    _sig(L, "rtm_bounds_probe", c_int, vp, vp, c_size, vp, c_size, I32P)
    _sig(L, "rtm_backward_normalized", c_int, vp, vp, vp, vp, vp, I32P, c_int, c_int, ctypes.c_float, vp, vp,
         c_int, I32P, vp)
    _sig(L, "rtm_plan_state_floats", c_size, vp)
    _sig(L, "rtm_plan_num_checkpoints", c_int, vp, c_int)
    _sig(L, "rtm_plan_checkpoint_bytes", c_size, vp, c_int, c_int)
    _sig(L, "rtm_forward_checkpointed", c_int, vp, vp, vp, c_int, c_int, vp, c_int, I32P, vp)
    _sig(L, "rtm_adjoint", c_int, vp, vp, vp, c_int, c_int, vp, vp, vp, vp)
    _sig(L, "rtm_backward_checkpointed", c_int, vp, vp, vp, c_int, c_int, vp, c_int, vp, vp, c_int, I32P, vp)
    _sig(L, "rtm_plan_set_callback", c_int, vp, c_int, STEP_CALLBACK, vp)
    _sig(L, "rtm_plan_wavefield", c_int, vp, c_int, vp, vp, vp, vp)
    for name, args in _OPTIONAL.items():
        if hasattr(L, name):
            _sig(L, name, *args)
    _lib = L
    return L


_OPTIONAL = {}


def check(code, fn):
    if code != 0:
        raise RtmError(code, fn)
    return code


def exported_symbols():
    """Names declared in include/rtm_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                       "rtm_b200.h")
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(rtm_\w+)\s*\(", text, re.M)))
