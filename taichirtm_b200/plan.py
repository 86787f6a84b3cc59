"""Python owner of an ``rtm_plan`` (include/rtm_b200.h): torch tensors for the
caller-side buffers, the C library for every kernel."""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import PSV, SH, BOTH, check  # noqa: F401

COL_OFF = 4


def _i32p(a):
    return a.ctypes.data_as(_lib.I32P)


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("taichirtm_b200 runs on a CUDA GPU (sm_100a); no CUDA device is visible")


class ShotGeometry:
    """One shot: window rows [x0, x0 + nx) of the global grid, LOCAL source and
    receiver grid indices (i, j)."""

    def __init__(self, x0, nx, src_ij, rec_ij):
        self.x0 = int(x0)
        self.nx = int(nx)
        self.src = np.ascontiguousarray(np.asarray(src_ij, np.int32).reshape(-1, 2))
        self.rec = np.ascontiguousarray(np.asarray(rec_ij, np.int32).reshape(-1, 2))


class Plan:
    """A set of shots on one grid, ready to propagate on the current device."""

    def __init__(self, nx, nz, dx, dz, nt, fs, absorbing_frame, modes, shots, tune=None,
                 device=None):
        require_cuda()
        self.device = torch.device(device if device is not None else "cuda")
        self.nx, self.nz, self.nt = int(nx), int(nz), int(nt)
        self.dx, self.dz, self.fs = float(dx), float(dz), float(fs)
        self.fw = int(absorbing_frame)
        self.modes = int(modes)
        self.shots = list(shots)
        self.nsrc = [len(s.src) for s in self.shots]
        self.nrec = [len(s.rec) for s in self.shots]
        self.nsrc_total = int(sum(self.nsrc))
        self.nrec_total = int(sum(self.nrec))
        L = _lib.lib()
        g = _lib.RtmGrid(self.nx, self.nz, self.dx, self.dz, self.fs, self.nt, self.fw, self.modes)
        arr = (_lib.RtmShot * len(self.shots))()
        self._keep = []
        for k, s in enumerate(self.shots):
            self._keep += [s.src, s.rec]
            arr[k] = _lib.RtmShot(s.x0, s.nx, len(s.src), _i32p(s.src), len(s.rec), _i32p(s.rec))
        t = tune or {}
        tn = _lib.RtmTune(int(t.get("vec", 0)), int(t.get("rows", 0)), int(t.get("warps", 0)),
                          int(t.get("prefetch", -1)), int(t.get("graphs", 0)), int(t.get("tsteps", 0)))
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(L.rtm_plan_create(ctypes.byref(g), len(self.shots), arr, ctypes.byref(tn),
                                    ctypes.byref(h)), "rtm_plan_create")
        self.h = h
        self.pitch = int(L.rtm_plan_pitch(h))
        self.rows_total = int(sum(s.nx for s in self.shots))
        self.model_set = False

    # ------------------------------------------------------------------ helpers
    def _f32(self, x, shape=None):
        t = torch.as_tensor(x) if not isinstance(x, torch.Tensor) else x
        t = t.to(device=self.device, dtype=torch.float32).contiguous()
        if shape is not None and tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
        return t

    def snapshot_buffer(self, nsnap):
        n = int(_lib.lib().rtm_plan_snapshot_floats(self.h, int(nsnap)))
        return torch.empty(max(n, 1), dtype=torch.float32, device=self.device)

    def launch_count(self):
        return int(_lib.lib().rtm_plan_launch_count(self.h))

    # ------------------------------------------------------------------ calls
    def set_model(self, mu, lam, rho, surface=None, stream=None):
        shp = (self.nx, self.nz)
        self._mu, self._lam, self._rho = (self._f32(x, shp) for x in (mu, lam, rho))
        self._surface = None if surface is None else self._f32(surface, shp)
        with torch.cuda.device(self.device):
            check(_lib.lib().rtm_plan_set_model(self.h, _ptr(self._mu), _ptr(self._lam),
                                                _ptr(self._rho), _ptr(self._surface),
                                                _stream(stream)), "rtm_plan_set_model")
        self.model_set = True

    def forward(self, wavelets, save=False, isnap=10, check_interval=100, stream=None,
                seis_out=None, snaps=None):
        """wavelets: (3, nsrc_total, nt).  Returns (flags, seis (3, nrec_total, nt),
        snaps [u, v, w] flat buffers or None, isnaps np.int32)."""
        wav = self._f32(wavelets, (3, self.nsrc_total, self.nt)) if self.nsrc_total else None
        seis = seis_out if seis_out is not None else torch.empty(
            (3, self.nrec_total, self.nt), dtype=torch.float32, device=self.device)
        nsnap = self.nt // int(isnap) if save else 0
        if save and snaps is None:
            snaps = [self.snapshot_buffer(nsnap) if self._comp_active(c) else None for c in range(3)]
        if not save:
            snaps = [None, None, None]
        isnaps = np.zeros(max(nsnap, 1), np.int32)
        flags = np.zeros(len(self.shots), np.int32)
        with torch.cuda.device(self.device):
            check(_lib.lib().rtm_forward(self.h, _ptr(wav), _ptr(seis), int(bool(save)), int(isnap),
                                         _ptr(snaps[0]), _ptr(snaps[1]), _ptr(snaps[2]), _i32p(isnaps),
                                         int(check_interval), _i32p(flags), _stream(stream)),
                  "rtm_forward")
        return flags, seis, (snaps if save else None), isnaps[:nsnap]

    def backward(self, obs, snaps, isnaps, num_snaps, isnap, check_interval=100, image=True,
                 stack=None, stream=None, normalize_eps=None):
        """obs: (3, nrec_total, nt).  Returns (flags, image (3, nx, nz) or None,
        stack (3, nx, nz) float64 or None).  normalize_eps (>= 0) selects the
        source-normalised cross-correlation: every shot's image divided by its
        source illumination + eps * its maximum (rtm_backward_normalized)."""
        o = self._f32(obs, (3, self.nrec_total, self.nt)) if self.nrec_total else None
        isn = np.ascontiguousarray(np.asarray(isnaps, np.int32).reshape(-1))
        if isn.size == 0:
            isn = np.zeros(1, np.int32)
        img = torch.empty((3, self.nx, self.nz), dtype=torch.float32, device=self.device) if image else None
        flags = np.zeros(len(self.shots), np.int32)
        snaps = snaps if snaps is not None else [None, None, None]
        with torch.cuda.device(self.device):
            if normalize_eps is None:
                check(_lib.lib().rtm_backward(self.h, _ptr(o), _ptr(snaps[0]), _ptr(snaps[1]),
                                              _ptr(snaps[2]), _i32p(isn), int(num_snaps), int(isnap),
                                              _ptr(img), _ptr(stack), int(check_interval), _i32p(flags),
                                              _stream(stream)), "rtm_backward")
            else:
                check(_lib.lib().rtm_backward_normalized(
                    self.h, _ptr(o), _ptr(snaps[0]), _ptr(snaps[1]), _ptr(snaps[2]), _i32p(isn), int(num_snaps),
                    int(isnap), float(normalize_eps), _ptr(img), _ptr(stack), int(check_interval), _i32p(flags),
                    _stream(stream)), "rtm_backward_normalized")
        return flags, img, stack

    def set_callback(self, forward_every, fn):
        """Host step callback (rtm_plan_set_callback): ``fn(step)`` after every
        forward step with step % forward_every == 0 and after every backward
        imaging step (its time t), with the live wavefield available through
        ``wavefield``.  A non-zero return (or an exception, re-raised by the
        caller) stops the loop.  ``fn`` None clears it."""
        L = _lib.lib()
        if fn is None:
            self._cb = None
            check(L.rtm_plan_set_callback(self.h, 0, _lib.STEP_CALLBACK(), None), "rtm_plan_set_callback")
            return
        self._cb = _lib.STEP_CALLBACK(lambda user, step: int(fn(int(step)) or 0))  # kept alive with the plan
        check(L.rtm_plan_set_callback(self.h, int(forward_every), self._cb, None), "rtm_plan_set_callback")

    def wavefield(self, shot=0, stream=None):
        """(3, nx_shot, nz) float32 device copy of the live u, v, w of one
        shot (rtm_plan_wavefield)."""
        s = self.shots[shot]
        out = torch.empty((3, s.nx, self.nz), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().rtm_plan_wavefield(self.h, int(shot), _ptr(out[0]), _ptr(out[1]), _ptr(out[2]),
                                                _stream(stream)), "rtm_plan_wavefield")
        return out

    def _comp_active(self, c):
        return bool(self.modes & SH) if c == 1 else bool(self.modes & PSV)

    def snapshot_view(self, buf, nsnap, shot=0):
        """(nx, nz, nsnap) view of one shot's snapshots (the reference's
        u_save_field shape, forward_modeling.py:533)."""
        s = self.shots[shot]
        off = sum(x.nx for x in self.shots[:shot]) * nsnap * self.pitch
        blk = buf[off: off + nsnap * s.nx * self.pitch].view(nsnap, s.nx, self.pitch)
        return blk[:, :, COL_OFF:COL_OFF + self.nz].permute(1, 2, 0)

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().rtm_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
