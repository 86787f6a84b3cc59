"""BackwardModeling with the reference's interface (src/backward_modeling.py),
run by the fused sm_100a kernels of librtm_b200."""
from typing import Callable, Optional

import numpy as np
import torch

from .fields import DeviceField, to_numpy, to_tensor
from .forward_modeling import material_is_regular, pick_modes, run_with_display
from .plan import PSV, SH, Plan, ShotGeometry, require_cuda


class BackwardModeling:
    """Time-reversed propagation with the zero-lag cross-correlation imaging
    condition (backward_modeling.py:32-77).  Same keyword arguments as the
    reference's constructor (backward_modeling.py:125-151)."""

    @staticmethod
    def estimate_memory_bytes(nx: int, nz: int, nt: int, num_sources: int, num_receivers: int) -> int:
        """Reference budget model (backward_modeling.py:79-123): 20 grid fields
        plus three (nsrc, nt) synthetic-source traces."""
        return 20 * nx * nz * 4 + 3 * num_sources * nt * 4

    def __init__(self, **kwargs):
        require_cuda()
        self.nx = kwargs["nx"]
        self.nz = kwargs["nz"]
        self.dx = float(kwargs["dx"])
        self.dz = float(kwargs["dz"])
        self.nt = kwargs["nt"]
        self.fs = float(kwargs["fs"])
        self.absorbing_frame = kwargs.get("absorbing_frame", 60)
        self.dt = 1.0 / self.fs
        self.num_sources = kwargs["num_sources"]
        self.num_receivers = kwargs["num_receivers"]
        self.device = torch.device(kwargs.get("device", "cuda"))
        dev = self.device
        self.src_loc_field = kwargs["src_loc_field"]
        self.recv_loc_field = kwargs["recv_loc_field"]
        self.obsdata_u_field = kwargs["obsdata_u_field"]
        self.obsdata_v_field = kwargs["obsdata_v_field"]
        self.obsdata_w_field = kwargs["obsdata_w_field"]
        self.surface_matrix = kwargs.get("surface_matrix_field", None)
        self._rec = to_numpy(self.recv_loc_field, np.int32).reshape(-1, 2)[: self.num_receivers]
        self.mu = to_tensor(kwargs["mu_field"], torch.float32, dev)
        self.lam = to_tensor(kwargs["lam_field"], torch.float32, dev)
        self.rho_field = to_tensor(kwargs["rho_field"], torch.float32, dev)
        obs = [to_tensor(o, torch.float32, dev).reshape(self.num_receivers, self.nt)
               for o in (self.obsdata_u_field, self.obsdata_v_field, self.obsdata_w_field)]
        self._obs = torch.stack(obs) if self.num_receivers else torch.zeros(3, 0, self.nt, device=dev)
        regular = material_is_regular(self.mu, self.lam, self.rho_field)
        self.modes = pick_modes(bool((obs[0] != 0).any() or (obs[2] != 0).any()) if obs else False,
                                bool((obs[1] != 0).any()) if obs else False, regular)
        self.tune = kwargs.get("tune", None)
        self._sm = None if self.surface_matrix is None else to_tensor(self.surface_matrix, torch.float32, dev)
        self.plan = None
        self._img = None

    def _make_plan(self, modes):
        if self.plan is not None and self.plan.modes == modes:
            return
        if self.plan is not None:
            self.plan.close()
        self.plan = Plan(self.nx, self.nz, self.dx, self.dz, self.nt, self.fs, self.absorbing_frame,
                         modes, [ShotGeometry(0, self.nx, np.zeros((0, 2), np.int32), self._rec)],
                         tune=self.tune, device=self.device)
        self.plan.set_model(self.mu, self.lam, self.rho_field, self._sm)

    def _snapshot_buffers(self, fw_fields, num_snaps):
        """Snapshot storage in the plan layout.  Fields produced by this
        package's ForwardModeling are used in place; anything else (NumPy,
        torch (nx, nz, nsnap), ti.field) is copied in once."""
        bufs = []
        for c, f in enumerate(fw_fields):
            active = bool(self.plan.modes & SH) if c == 1 else bool(self.plan.modes & PSV)
            if not active or num_snaps <= 0:
                bufs.append(None)
                continue
            owner = getattr(f, "_owner", None) if isinstance(f, DeviceField) else None
            if owner is not None and owner.numel() >= self.plan.rows_total * self.plan.pitch * num_snaps \
                    and getattr(f, "tensor", None) is not None and tuple(f.shape) == (self.nx, self.nz, num_snaps) \
                    and f.tensor.stride()[0] == self.plan.pitch:
                bufs.append(owner)
                continue
            t = to_tensor(f, torch.float32, self.device).reshape(self.nx, self.nz, -1)[:, :, :num_snaps]
            buf = self.plan.snapshot_buffer(num_snaps)
            self.plan.snapshot_view(buf, num_snaps).copy_(t)
            bufs.append(buf)
        return bufs

    def run_calc(self, import_fwdata_u, import_fwdata_v, import_fwdata_w, isnaps_field,
                 num_snaps: int, isnap_interval: int, method: str = "cross_correlation",
                 display_callback: Optional[Callable] = None,
                 stability_check_interval: int = 100, *, normalization_eps: float = 1e-3) -> int:
        """BackwardModeling.run_calc (backward_modeling.py:498-579): 0 on
        success, 4 / 5 / 6 when u / v / w became non-finite.

        ``method``: "cross_correlation" (default) and any name the reference
        accepts without using it ("convolution", bm:505) give the reference's
        zero-lag cross-correlation; "source_normalized" (an extension) divides
        the image by the source illumination sum_t snapshot^2 plus
        ``normalization_eps`` times its maximum."""
        self._make_plan(self.modes)
        isnaps = to_numpy(isnaps_field, np.int32).reshape(-1)[: max(int(num_snaps), 0)]
        snaps = self._snapshot_buffers((import_fwdata_u, import_fwdata_v, import_fwdata_w), int(num_snaps))
        eps = float(normalization_eps) if method == "source_normalized" else None

        def run():
            flags, img, _ = self.plan.backward(self._obs, snaps, isnaps, int(num_snaps), int(isnap_interval),
                                               check_interval=stability_check_interval, image=True,
                                               normalize_eps=eps)
            self._img = img
            return int(flags[0])
        if display_callback is None:
            return run()
        # like the reference (backward_modeling.py:565-569): the live backward
        # wavefield after every imaging step, with its time t
        return run_with_display(self.plan, 0, display_callback, self.dx, self.dz, run)

    def get_results(self) -> tuple:
        """(image_u, image_v, image_w), each (nx, nz) float32 NumPy."""
        if self._img is None:
            z = np.zeros((self.nx, self.nz), np.float32)
            return z, z.copy(), z.copy()
        a = self._img.cpu().numpy()
        return a[0].copy(), a[1].copy(), a[2].copy()

    def get_result_tensors(self):
        return self._img

    def cleanup(self):
        """Release device memory held by this instance (backward_modeling.py:589-645)."""
        if self.plan is not None:
            self.plan.close()
            self.plan = None
        for name in ("_img", "_obs", "mu", "lam", "rho_field", "_sm", "src_loc_field", "recv_loc_field",
                     "obsdata_u_field", "obsdata_v_field", "obsdata_w_field", "surface_matrix"):
            if hasattr(self, name):
                setattr(self, name, None)
