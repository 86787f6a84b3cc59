"""Batched RTM: many shots, each on its own window of one model, advanced
together -- one kernel launch per time step covers every shot.

The reference runs one shot per ``ReverseTimeMigration.run`` and sums the
per-shot images afterwards (examples/example_2nd_step.py:102-158,
src/imaging.py:81-93).  Here each shot keeps the reference's semantics on its
window (a window behaves exactly like the reference run on the cropped model:
sponge, edge cells and injection use the window's own edges), and the
cross-shot sum is an FP64 reduction on the GPU."""
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib, autotune
from .fields import to_tensor
from .plan import PSV, SH, Plan, ShotGeometry, _i32p, _ptr, _stream, check, require_cuda


class _StreamedTensor:
    """A device tensor being filled on a side stream: ``get()`` makes the
    current stream wait for that copy, then returns the tensor."""

    def __init__(self, t, stream):
        self.t, self.event = t, torch.cuda.Event()
        self.event.record(stream)

    def get(self):
        torch.cuda.current_stream(self.t.device).wait_event(self.event)
        return self.t


def _ready(x):
    return x.get() if isinstance(x, _StreamedTensor) else x


class BatchedRTM:
    """Many shots on one model.

    mu, lam, rho : (nx, nz) model (the reference's mu/lam/rho fields).
    shots        : ShotGeometry list (window rows and LOCAL source/receiver
                   grid indices).
    modes        : PSV, SH or BOTH (default PSV).
    tune         : launch shape dict, "auto" (autotuner, cached), or None.
    """

    def __init__(self, mu, lam, rho, dx, dz, fs, nt, absorbing_frame, shots: Sequence[ShotGeometry],
                 modes=PSV, surface=None, tune="auto", device=None, graphs=True):
        require_cuda()
        self.device = torch.device(device if device is not None else "cuda")
        self.nx, self.nz = tuple(np.shape(mu))
        self.dx, self.dz, self.fs, self.nt = float(dx), float(dz), float(fs), int(nt)
        self.fw = int(absorbing_frame)
        self.modes = int(modes)
        self.shots: List[ShotGeometry] = list(shots)
        self._model = [to_tensor(x, torch.float32, self.device) for x in (mu, lam, rho)]
        self._surface = None if surface is None else to_tensor(surface, torch.float32, self.device)
        if tune == "auto":
            tune = autotune.best_shape(self._make_plan, self.nz, self.shots, self.modes, self.nt)
        # time loops replayed as CUDA graphs: repeated calls on the same buffers
        # skip the per-step launch overhead
        tune = dict(tune or {}, graphs=int(bool(graphs)))
        self.tune = tune
        self.plan = self._make_plan(tune, self.nt)

    def _make_plan(self, tune, nt):
        p = Plan(self.nx, self.nz, self.dx, self.dz, nt, self.fs, self.fw, self.modes, self.shots,
                 tune=tune, device=self.device)
        p.set_model(*self._model, self._surface)
        return p

    @property
    def nsrc_total(self):
        return self.plan.nsrc_total

    @property
    def nrec_total(self):
        return self.plan.nrec_total

    def cells(self):
        return sum(s.nx for s in self.shots) * self.nz

    def forward(self, wavelets, save=False, isnap=10, check_interval=100):
        """wavelets (3, nsrc_total, nt) -> (flags, seismograms (3, nrec_total, nt),
        snapshot buffers, isnaps)."""
        w = to_tensor(wavelets, torch.float32, self.device)
        return self.plan.forward(w, save=save, isnap=isnap, check_interval=check_interval)

    def migrate(self, wavelets, observed, isnap=10, check_interval=100, stack=None, checkpoint=None,
                method="cross_correlation", normalization_eps=1e-3):
        """Forward with snapshots, backward with imaging, FP64 stack of every
        shot's image on the global grid.  Returns (forward flags, backward
        flags, stack (3, nx, nz) float64 on the device).

        ``checkpoint=dict(every=K, dtype="f32"|"f16"|"bf16")`` stores the full
        wavefield every K steps instead of snapshots and recomputes the
        forward wavefield segment by segment during the backward pass (P-SV):
        memory ~ (nt/K) x 5 fields instead of (nt/isnap) x 2, one extra
        forward pass of compute; FP32 checkpoints give the same image bits.

        ``method="source_normalized"`` divides every shot's image by its source
        illumination (sum of squared snapshots over the imaging steps) plus
        ``normalization_eps`` times its maximum before stacking (snapshot path).

        ``observed`` may be a pinned host float32 tensor: it is then copied
        to the device on a side stream while the forward pass runs (only the
        backward pass reads it)."""
        w = to_tensor(wavelets, torch.float32, self.device)
        o = self._observed_async(observed)
        if checkpoint:
            if method == "source_normalized":
                raise ValueError("source_normalized imaging needs the snapshot path (checkpoint=None)")
            return self._migrate_checkpointed(w, o, isnap, check_interval, stack, checkpoint)
        ff, _, snaps, isnaps = self.plan.forward(w, save=True, isnap=isnap, check_interval=check_interval)
        if stack is None:
            stack = torch.zeros((3, self.nx, self.nz), dtype=torch.float64, device=self.device)
        o = _ready(o)
        fb, _, _ = self.plan.backward(o, snaps, isnaps, len(isnaps), isnap, check_interval=check_interval,
                                      image=False, stack=stack,
                                      normalize_eps=normalization_eps if method == "source_normalized" else None)
        del snaps
        return ff, fb, stack

    def _observed_async(self, observed):
        """Device copy of ``observed``; a pinned contiguous float32 host tensor
        goes over on a side stream, and the current stream waits for it only
        when the copy is first used, i.e. before the backward pass."""
        if not (isinstance(observed, torch.Tensor) and observed.device.type == "cpu" and observed.is_pinned()
                and observed.dtype == torch.float32 and observed.is_contiguous()):
            return to_tensor(observed, torch.float32, self.device)
        main = torch.cuda.current_stream(self.device)
        side = getattr(self, "_copy_stream", None)
        if side is None:
            side = self._copy_stream = torch.cuda.Stream(device=self.device)
        side.wait_stream(main)  # the destination's previous users are done
        with torch.cuda.stream(side):
            dst = torch.empty(observed.shape, dtype=torch.float32, device=self.device)
            dst.copy_(observed, non_blocking=True)
        dst.record_stream(main)
        return _StreamedTensor(dst, side)

    def checkpoint_bytes(self, every, dtype="f32"):
        return int(_lib.lib().rtm_plan_checkpoint_bytes(self.plan.h, int(every), _lib.CKPT_DTYPES[dtype]))

    def _migrate_checkpointed(self, w, o, isnap, check_interval, stack, checkpoint):
        every = int(checkpoint.get("every") or max(1, round(self.nt ** 0.5)))
        dt = _lib.CKPT_DTYPES[checkpoint.get("dtype", "f32")]
        L = _lib.lib()
        ck = torch.empty(max(int(L.rtm_plan_checkpoint_bytes(self.plan.h, every, dt)), 1), dtype=torch.uint8,
                         device=self.device)
        seis = torch.empty((3, self.plan.nrec_total, self.nt), dtype=torch.float32, device=self.device)
        ff = np.zeros(len(self.shots), np.int32)
        fb = np.zeros(len(self.shots), np.int32)
        if stack is None:
            stack = torch.zeros((3, self.nx, self.nz), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(L.rtm_forward_checkpointed(self.plan.h, _ptr(w), _ptr(seis), every, dt, _ptr(ck),
                                             int(check_interval), _i32p(ff), _stream()), "rtm_forward_checkpointed")
            o = _ready(o)
            check(L.rtm_backward_checkpointed(self.plan.h, _ptr(w), _ptr(o), every, dt, _ptr(ck), int(isnap), None,
                                              _ptr(stack), int(check_interval), _i32p(fb), _stream()),
                  "rtm_backward_checkpointed")
        return ff, fb, stack

    def launch_count(self):
        return self.plan.launch_count()

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None


def survey_shots(survey) -> List[ShotGeometry]:
    """ShotGeometry list of a taichirtm_b200.synthetic.Survey."""
    return [ShotGeometry(s.x0, s.nx, s.src, s.rec) for s in survey.shots]


def survey_wavelets(survey) -> np.ndarray:
    return np.concatenate([s.wavelets for s in survey.shots], axis=1)


def modes_of(name: Optional[str]):
    return {"psv": PSV, "sh": SH, "both": PSV | SH}[name or "psv"]
