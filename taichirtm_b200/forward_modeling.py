"""ForwardModeling with the reference's interface (src/forward_modeling.py), run
by the fused sm_100a kernels of librtm_b200."""
from typing import Callable, Optional

import numpy as np
import torch

from .fields import DeviceField, to_numpy, to_tensor
from .plan import BOTH, PSV, SH, Plan, ShotGeometry, require_cuda


def material_is_regular(mu, lam, rho):
    """True when every derived coefficient is finite on the interior, so a
    mode with zero sources stays exactly zero and may be skipped."""
    return bool(torch.isfinite(mu).all() and torch.isfinite(lam).all() and torch.isfinite(rho).all()
                and (mu > 0).all() and (rho > 0).all())


def pick_modes(psv_sources, sh_sources, regular):
    """The reference always advances P-SV and SH together; the two never read
    each other's fields (forward_modeling.py:330-384), so a mode whose sources
    are all zero stays zero and can be skipped without changing any output,
    provided the material is regular (no 0/0 averages that would turn a zero
    field into NaN)."""
    if not regular:
        return BOTH
    m = (PSV if psv_sources else 0) | (SH if sh_sources else 0)
    return m or PSV


def run_with_display(plan, every, display_callback, dx, dz, run):
    """Run ``run()`` with the plan's step callback calling
    display_callback(u, v, w, step, nx, nz, dx, dz) with host copies of shot
    0's live wavefield (forward: every ``every`` steps; backward: at the
    imaging steps).  An exception in display_callback stops the time loop and
    is re-raised."""
    from ._lib import RtmError
    nx, nz = plan.shots[0].nx, plan.nz
    err = []

    def cb(step):
        try:
            f = plan.wavefield(0).cpu().numpy()
            display_callback(f[0], f[1], f[2], step, nx, nz, dx, dz)
            return 0
        except BaseException as e:  # noqa: BLE001 - re-raised after the C call returns
            err.append(e)
            return 1
    plan.set_callback(every, cb)
    try:
        return run()
    except RtmError:
        if err:
            raise err[0]
        raise
    finally:
        plan.set_callback(0, None)


class ForwardModeling:
    """Forward modeling of P-SV and SH waves (forward_modeling.py:32-79).

    Same keyword arguments as the reference's constructor
    (forward_modeling.py:126-153); fields may be torch tensors, NumPy arrays or
    objects with ``to_numpy()``."""

    @staticmethod
    def estimate_memory_bytes(nx: int, nz: int, nt: int, num_sources: int, num_receivers: int) -> int:
        """Same budget model as the reference (forward_modeling.py:81-124): 17
        (nx, nz) float32 grid fields plus three (nrec, nt) seismograms.  Used by
        ReverseTimeMigration._compute_isnap so the snapshot interval matches."""
        return 17 * nx * nz * 4 + 3 * num_receivers * nt * 4

    def __init__(self, **kwargs):
        require_cuda()
        self.nx = kwargs["nx"]
        self.nz = kwargs["nz"]
        self.dx = float(kwargs["dx"])
        self.dz = float(kwargs["dz"])
        self.nt = kwargs["nt"]
        self.fs = float(kwargs["fs"])
        self.absorbing_frame = kwargs.get("absorbing_frame", 60)
        self.isnap = kwargs.get("isnap", 10)
        self.dt = 1.0 / self.fs
        self.num_sources = kwargs["num_sources"]
        self.num_receivers = kwargs["num_receivers"]
        self.device = torch.device(kwargs.get("device", "cuda"))
        dev = self.device
        self.src_loc_field = kwargs["src_loc_field"]
        self.recv_loc_field = kwargs["recv_loc_field"]
        self.wavelet_u_field = kwargs["wavelet_u_field"]
        self.wavelet_v_field = kwargs["wavelet_v_field"]
        self.wavelet_w_field = kwargs["wavelet_w_field"]
        self.surface_matrix = kwargs.get("surface_matrix_field", None)
        src = to_numpy(self.src_loc_field, np.int32).reshape(-1, 2)[: self.num_sources]
        rec = to_numpy(self.recv_loc_field, np.int32).reshape(-1, 2)[: self.num_receivers]
        self.mu = to_tensor(kwargs["mu_field"], torch.float32, dev)
        self.lam = to_tensor(kwargs["lam_field"], torch.float32, dev)
        self.rho_field = to_tensor(kwargs["rho_field"], torch.float32, dev)
        wav = [to_tensor(w, torch.float32, dev).reshape(self.num_sources, self.nt)
               for w in (self.wavelet_u_field, self.wavelet_v_field, self.wavelet_w_field)]
        self._wavelets = torch.stack(wav) if self.num_sources else torch.zeros(3, 0, self.nt, device=dev)
        edge = bool(((src[:, 0] <= 0) | (src[:, 0] >= self.nx - 1) | (src[:, 1] <= 0)
                     | (src[:, 1] >= self.nz - 1)).any()) if len(src) else False
        regular = material_is_regular(self.mu, self.lam, self.rho_field)
        psv = edge or bool((wav[0] != 0).any() or (wav[2] != 0).any())
        sh = bool((wav[1] != 0).any())
        self.modes = pick_modes(psv, sh, regular)
        self.tune = kwargs.get("tune", None)
        self.plan = Plan(self.nx, self.nz, self.dx, self.dz, self.nt, self.fs, self.absorbing_frame,
                         self.modes, [ShotGeometry(0, self.nx, src, rec)], tune=self.tune, device=dev)
        sm = None if self.surface_matrix is None else to_tensor(self.surface_matrix, torch.float32, dev)
        self.plan.set_model(self.mu, self.lam, self.rho_field, sm)
        self._seis = None
        self.num_snaps = 0

    def run(self, save: bool = False, display_callback: Optional[Callable] = None,
            stability_check_interval: int = 100) -> int:
        """ForwardModeling.run (forward_modeling.py:504-575): 0 on success,
        1 / 2 / 3 when u / v / w became non-finite (highest code wins)."""
        if display_callback is not None:
            return self._run_with_callback(save, display_callback, stability_check_interval)
        return self._run_plain(save, stability_check_interval)

    def _expose_snapshots(self, snaps, isnaps):
        n = self.nt // self.isnap
        self.num_snaps = n
        self._snap_buffers = snaps
        views = []
        for c in range(3):
            if snaps[c] is None:
                views.append(DeviceField(torch.zeros((self.nx, self.nz, n), device=self.device)))
            else:
                views.append(DeviceField(self.plan.snapshot_view(snaps[c], n), owner=snaps[c]))
        self.u_save_field, self.v_save_field, self.w_save_field = views
        self.isnaps_field = DeviceField(torch.as_tensor(np.asarray(isnaps, np.int32), device=self.device))
        self._snap_plan_pitch = self.plan.pitch

    def _run_with_callback(self, save, display_callback, stability_check_interval):
        """Callback path: like the reference (forward_modeling.py:553-559),
        display_callback(u, v, w, it, nx, nz, dx, dz) receives host copies of
        the live wavefield after every step with it % isnap == 0, it = 0
        included, during the run; no callback follows a failed finite check.
        The time loop then runs as direct launches ending at those steps."""
        return run_with_display(self.plan, self.isnap, display_callback, self.dx, self.dz,
                                lambda: self._run_plain(save, stability_check_interval))

    def _run_plain(self, save, stability_check_interval):
        flags, seis, snaps, isnaps = self.plan.forward(self._wavelets, save=save, isnap=self.isnap,
                                                       check_interval=stability_check_interval)
        self._seis = seis
        if save:
            self._expose_snapshots(snaps, isnaps)
        return int(flags[0])

    def get_seismogram(self) -> tuple:
        """(u, v, w) seismograms, each (num_receivers, nt) float32 NumPy."""
        if self._seis is None:
            z = np.zeros((self.num_receivers, self.nt), np.float32)
            return z, z.copy(), z.copy()
        s = self._seis.cpu().numpy()
        return s[0].copy(), s[1].copy(), s[2].copy()

    def get_seismogram_tensors(self):
        """Device-resident (3, nrec, nt) seismograms (no host copy)."""
        return self._seis

    def cleanup(self):
        """Release device memory held by this instance (forward_modeling.py:585-646)."""
        if getattr(self, "plan", None) is not None:
            self.plan.close()
            self.plan = None
        for name in ("u_save_field", "v_save_field", "w_save_field", "isnaps_field", "_snap_buffers",
                     "_seis", "_wavelets", "mu", "lam", "rho_field", "src_loc_field", "recv_loc_field",
                     "wavelet_u_field", "wavelet_v_field", "wavelet_w_field", "surface_matrix"):
            if hasattr(self, name):
                setattr(self, name, None)
