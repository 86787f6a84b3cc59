"""ReverseTimeMigration with the reference's interface (src/rtm.py), driving the
GPU ForwardModeling / BackwardModeling of this package.

The orchestration (validation, velocity scan, grid and material set-up,
topography mask, memory-budgeted snapshot interval, CFL-halving retry, npz
output) keeps the reference's rules; only the propagation runs differently."""
import os
import warnings
from typing import Callable, Optional

import numpy as np
import torch

from .backward_modeling import BackwardModeling
from .forward_modeling import ForwardModeling

_BACKENDS = ("cpu", "gpu", "cuda", "vulkan", "opengl", "metal")
_state = {"device": None}


def reset_taichi():
    """rtm.py:43-53 released every Taichi field; here it releases the CUDA
    caching allocator's unused blocks (plans free their own memory)."""
    if torch.cuda.is_available():
        torch.cuda.synchronize()
        torch.cuda.empty_cache()


def init_taichi(backend: str = "cpu", extreme_optimization: bool = False, **kwargs):
    """rtm.py:56-133 selected a Taichi arch.  This package has one backend,
    hand-written sm_100a CUDA, so every backend name selects the CUDA device
    (``device_index`` kwarg, default the current one).  Non-GPU names are
    accepted for drop-in compatibility and announced with a warning."""
    b = str(backend).lower()
    if b not in ("gpu", "cuda"):
        warnings.warn(f"backend '{backend}' requested: taichirtm_b200 always runs on the CUDA GPU",
                      RuntimeWarning, stacklevel=2)
    if not torch.cuda.is_available():
        raise RuntimeError("taichirtm_b200 needs a CUDA GPU; none is visible")
    idx = kwargs.get("device_index", torch.cuda.current_device())
    torch.cuda.set_device(idx)
    _state["device"] = torch.device("cuda", idx)
    return _state["device"]


class ReverseTimeMigration:
    """Reverse Time Migration (rtm.py:136-205): fluent API and the deprecated
    kwargs constructor, same defaults."""

    def __init__(self, **kwargs):
        self.observed_u = None
        self.observed_v = None
        self.observed_w = None
        self.source_u = None
        self.source_v = None
        self.source_w = None
        self.receiver_loc = None
        self.receiver_num = None
        self.source_loc = None
        self.fs = None
        self.nt = None
        self.rho = 1500
        self.poisson = 0.33
        self.isnap = 216
        self.absorbing_frame = 50
        self.vmin = 10.0
        self.vmax = 500.0
        self.vstep = 10
        self.v_fix = None
        self.total_allocate_memory_gb = 8.0
        self.receivers_height = None
        self.debug = False
        self._fw_instance = None
        self._bw_instance = None
        self._run_fields = []
        if kwargs:
            warnings.warn(
                "The kwargs-based constructor is deprecated. "
                "Please use the fluent API (set_observed_data, set_source, etc.) instead.",
                DeprecationWarning, stacklevel=2)
            self._init_from_kwargs(kwargs)

    def _init_from_kwargs(self, kwargs):
        """rtm.py:249-284."""
        self.observed_u = np.asarray(kwargs["observed_u"], dtype=np.float32)
        self.observed_v = np.asarray(kwargs["observed_v"], dtype=np.float32)
        self.observed_w = np.asarray(kwargs["observed_w"], dtype=np.float32)
        self.source_u = np.asarray(kwargs["source_u"], dtype=np.float32)
        self.source_v = np.asarray(kwargs["source_v"], dtype=np.float32)
        self.source_w = np.asarray(kwargs["source_w"], dtype=np.float32)
        self.receiver_loc = np.asarray(kwargs["receiver_loc"], dtype=np.float32)
        self.receiver_num = len(self.receiver_loc)
        self.source_loc = float(kwargs["source_loc"])
        self.fs = float(kwargs["fs"])
        self.rho = kwargs.get("rho", 1500)
        self.poisson = kwargs.get("poisson_ratio", 0.33)
        self.isnap = kwargs.get("isnap", 216)
        self.nt = self.observed_u.shape[1]
        self.absorbing_frame = kwargs.get("absorbing_frame", 50)
        self.vmin = kwargs.get("vmin", 10.0)
        self.vmax = kwargs.get("vmax", 500.0)
        self.vstep = kwargs.get("vstep", 10)
        self.v_fix = kwargs.get("v_fix", None)
        self.total_allocate_memory_gb = kwargs.get("total_allocate_memory_gb", 8.0)
        self.receivers_height = kwargs.get("receivers_height", None)
        if self.receivers_height is not None:
            self.receivers_height = np.asarray(self.receivers_height, dtype=np.float32)
            self.receivers_height = self.receivers_height - np.max(self.receivers_height)
        self._check_parameters()

    # ------------------------------------------------------------ context manager
    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_val, exc_tb):
        self.cleanup()
        return False

    def cleanup(self, reset_taichi_runtime: bool = True):
        """rtm.py:297-328."""
        if self._fw_instance is not None:
            self._fw_instance.cleanup()
            self._fw_instance = None
        if self._bw_instance is not None:
            self._bw_instance.cleanup()
            self._bw_instance = None
        self._run_fields.clear()
        if reset_taichi_runtime:
            reset_taichi()

    # ------------------------------------------------------------ fluent setters (rtm.py:332-561)
    def set_observed_data(self, observed_u, observed_v, observed_w):
        self.observed_u = np.asarray(observed_u, dtype=np.float32)
        self.observed_v = np.asarray(observed_v, dtype=np.float32)
        self.observed_w = np.asarray(observed_w, dtype=np.float32)
        self.nt = self.observed_u.shape[1]
        return self

    def set_source(self, source_u, source_v, source_w, source_loc):
        self.source_u = np.asarray(source_u, dtype=np.float32)
        self.source_v = np.asarray(source_v, dtype=np.float32)
        self.source_w = np.asarray(source_w, dtype=np.float32)
        self.source_loc = float(source_loc)
        return self

    def set_receivers(self, receiver_loc):
        self.receiver_loc = np.asarray(receiver_loc, dtype=np.float32)
        self.receiver_num = len(self.receiver_loc)
        return self

    def set_frequency(self, fs):
        self.fs = float(fs)
        return self

    def set_velocity_range(self, vmin, vmax, vstep):
        self.vmin = float(vmin)
        self.vmax = float(vmax)
        self.vstep = int(vstep)
        return self

    def fix_velocity(self, velocity):
        self.v_fix = float(velocity)
        return self

    def set_boundary(self, absorbing_frame):
        self.absorbing_frame = int(absorbing_frame)
        return self

    def set_memory(self, total_allocate_memory_gb):
        self.total_allocate_memory_gb = float(total_allocate_memory_gb)
        return self

    def set_density(self, rho):
        self.rho = float(rho)
        return self

    def set_poisson_ratio(self, poisson_ratio):
        self.poisson = float(poisson_ratio)
        return self

    def set_topography(self, receivers_height):
        self.receivers_height = np.asarray(receivers_height, dtype=np.float32)
        self.receivers_height = self.receivers_height - np.max(self.receivers_height)
        return self

    def set_debug(self, debug: bool = True):
        self.debug = debug
        return self

    def _check_parameters(self):
        """rtm.py:563-601, same messages."""
        if self.observed_u is None or self.observed_v is None or self.observed_w is None:
            raise ValueError("Observed data must be provided. "
                             "Use set_observed_data(observed_u, observed_v, observed_w) to set it.")
        if self.source_u is None or self.source_v is None or self.source_w is None:
            raise ValueError("Source functions must be provided. "
                             "Use set_source(source_u, source_v, source_w, source_loc) to set them.")
        if self.receiver_loc is None:
            raise ValueError("Receiver locations must be provided. "
                             "Use set_receivers(receiver_loc) to set them.")
        if self.source_loc is None:
            raise ValueError("Source location must be provided. "
                             "Use set_source(source_u, source_v, source_w, source_loc) to set it.")
        if self.fs is None:
            raise ValueError("Sampling frequency must be provided. Use set_frequency(fs) to set it.")
        if self.observed_u.shape != self.observed_v.shape or self.observed_u.shape != self.observed_w.shape:
            raise ValueError("Observed data shapes must match")
        if self.source_u.shape != self.source_v.shape or self.source_u.shape != self.source_w.shape:
            raise ValueError("Source function shapes must match")
        if self.fs <= 0:
            raise ValueError("Sampling frequency must be positive")
        if self.receivers_height is not None:
            if len(self.receivers_height) != self.receiver_num:
                raise ValueError("Receiver height array size must match receiver count")

    def estimate_velocity(self, array: np.ndarray, vmin: float, vmax: float, vstep: int = 10) -> float:
        """Velocity scan of rtm.py:603-652: for each of ``vstep`` geometrically
        spaced trial velocities, shift every trace by its rounded moveout
        fs*|x_r - x_s|/v (relative to the smallest), multiply the aligned
        traces sample by sample, and keep the velocity with the largest
        |sum of products| (the first one on ties; vmin if none is positive)."""
        print("Estimating velocity...")
        nrec, nsamp = array.shape
        ratio = (vmax / vmin) ** (1 / (vstep - 1))
        dist = np.abs(self.receiver_loc - self.source_loc)
        best_v, best_score = vmin, 0
        for v in vmin * ratio ** np.arange(vstep):
            lag = np.round(self.fs * dist / v).astype(np.int32)
            lag = lag - lag.min()
            span = nsamp - lag.max()
            if span <= 0:
                continue
            aligned = np.take_along_axis(array, lag[:, None] + np.arange(span)[None, :], axis=1)
            score = np.abs(np.sum(np.prod(aligned, axis=0)))
            if score > best_score:
                best_v, best_score = v, score
        print(f"Estimated velocity: {best_v:.2f} m/s")
        return float(best_v)

    def _setup_modeling_conditions(self, estimated_v: float, CFL: float, absorbing_frame: int):
        """Homogeneous square model of rtm.py:654-666: dx = dz = v / fs / CFL,
        nx = nz = int(receiver span / dx) + 4 FW, constant rho and vs, vp from
        Poisson's ratio."""
        dx = estimated_v / self.fs / CFL
        span = np.max(self.receiver_loc) - np.min(self.receiver_loc)
        n = int(span / dx) + 4 * absorbing_frame
        rho = np.full((n, n), self.rho, dtype=np.float32)
        vs = np.full((n, n), estimated_v, dtype=np.float32)
        vp = (np.sqrt((2 * self.poisson + 1) / (1 - 2 * self.poisson)) * vs).astype(np.float32)
        return dx, dx, n, n, rho, vs, vp

    def _setup_surface_and_locations(self, nx, nz, dx, dz, absorbing_frame):
        """Grid positions and topography of rtm.py:668-717.

        Receivers and the source sit at column int(x / dx + 2 FW), row 1.  With
        receiver heights, each receiver moves to row int(-h / dz); the surface
        row between receivers is the truncated linear interpolation of the
        (float) receiver rows, flat before the first and after the last
        receiver; cells above it get mask 0; the source goes one row below the
        surface at its column."""
        pad = 2 * absorbing_frame
        rec = [[int(x / dx + pad), 1] for x in self.receiver_loc]
        src = [[int(self.source_loc / dx + pad), 1]]
        mask = np.ones((nx, nz), dtype=np.float32)
        surf_row = np.zeros(nx, dtype=np.float32)
        if self.receivers_height is None:
            self.surface_matrix = None
            return rec, src, mask
        rows_f = -1 * self.receivers_height / dz
        for n in range(len(rec)):
            rec[n][1] = int(rows_f[n])
        first_col, first_row = rec[0]
        mask[:first_col, :first_row] = 0
        surf_row[:first_col] = first_row
        for n in range(1, len(rec)):
            c_a, c_b = rec[n - 1][0], rec[n][0]
            h_a, h_b = rows_f[n - 1], rows_f[n]
            for col in range(c_a, c_b):
                h = int((h_b - h_a) / (c_b - c_a) * (col - c_a) + h_a)
                mask[col, :h] = 0
                surf_row[col] = h
        last_col = rec[-1][0]
        surf_row[last_col:] = rows_f[-1]
        mask[last_col:, :int(rows_f[-1])] = 0
        src[0][1] = int(surf_row[src[0][0]]) + 1
        self.height_array = surf_row
        self.surface_matrix = mask
        return rec, src, mask

    def _compute_isnap(self, nx: int, nz: int, nt: int, num_sources: int, num_receivers: int) -> int:
        """Snapshot interval from the memory budget, rtm.py:719-844, so that
        snapshots are taken at the same steps as the reference.

        Budget = total_allocate_memory_gb GiB minus 5 %; fixed part = 300 MiB
        runtime + inputs (3 material grids, locations, 3 wavelets, surface
        grid) + ForwardModeling and BackwardModeling estimates + 3 observed
        traces; each snapshot index costs 2 x 3 grids plus one int.  isnap =
        ceil(nt / max snapshots), 1 when everything fits, nt when nothing does."""
        f4 = 4
        budget = int(self.total_allocate_memory_gb * 1024 * 1024 * 1024)
        grid = nx * nz * f4
        inputs = 3 * grid + (2 * num_sources + 2 * num_receivers) * f4 \
            + 3 * num_sources * nt * f4 + grid
        fixed = (300 * 1024 * 1024 + inputs
                 + ForwardModeling.estimate_memory_bytes(nx, nz, nt, num_sources, num_receivers)
                 + 3 * num_receivers * nt * f4
                 + BackwardModeling.estimate_memory_bytes(nx, nz, nt, num_sources, num_receivers))
        room = budget - fixed - int(budget * 0.05)
        if room <= 0:
            print(f"Warning: Very limited memory available ({self.total_allocate_memory_gb:.1f} GB), "
                  "using minimum snapshots")
            return nt
        per_snapshot = 2 * 3 * grid + f4
        max_snaps = room // per_snapshot
        if max_snaps <= 0:
            return nt
        if max_snaps >= nt:
            return 1
        isnap = max(1, int(np.ceil(nt / max_snaps)))
        if self.debug:
            k = nt // isnap
            print(f"Snapshots: {k} x {per_snapshot / 2**20:.1f} MiB, isnap={isnap}, "
                  f"fixed {fixed / 2**30:.2f} GiB of {budget / 2**30:.2f} GiB")
        return isnap

    def run(self, method: str = "cross_correlation", display_callback: Optional[Callable] = None):
        """rtm.py:846-1029: forward with snapshots, backward with imaging; on a
        non-finite flag the CFL number is halved and the grid rebuilt."""
        self._check_parameters()
        if self.v_fix is not None:
            print(f"Using fixed velocity: {self.v_fix} m/s")
            estimated_v = self.v_fix
        else:
            estimated_v = self.estimate_velocity(self.observed_v, self.vmin, self.vmax, self.vstep)
        CFL = 0.8
        absorbing_frame = self.absorbing_frame
        flag = 99
        print("\nStarting forward modeling...")
        device = _state["device"] or torch.device("cuda")
        while flag:
            CFL *= 0.5
            flag = 0
            dx, dz, nx, nz, rho, vs, vp = self._setup_modeling_conditions(estimated_v, CFL, absorbing_frame)
            receiver_loc_step, src_loc_step, surface_matrix = self._setup_surface_and_locations(
                nx, nz, dx, dz, absorbing_frame)
            wavelet_u = self.source_u.reshape(1, -1) if self.source_u.ndim == 1 else self.source_u
            wavelet_v = self.source_v.reshape(1, -1) if self.source_v.ndim == 1 else self.source_v
            wavelet_w = self.source_w.reshape(1, -1) if self.source_w.ndim == 1 else self.source_w
            num_sources = len(src_loc_step)
            num_receivers = len(receiver_loc_step)
            isnap = self._compute_isnap(nx, nz, self.nt, num_sources, num_receivers)
            mu_np = (rho * vs ** 2).astype(np.float32)                   # rtm.py:901
            lam_np = (((vp / vs) ** 2 - 2) * mu_np).astype(np.float32)   # rtm.py:902
            src_np = np.array(src_loc_step, dtype=np.int32)
            rec_np = np.array(receiver_loc_step, dtype=np.int32)
            sm = None if self.surface_matrix is None else np.asarray(surface_matrix, np.float32)
            fw = ForwardModeling(
                nx=nx, nz=nz, dx=dx, dz=dz, nt=self.nt, fs=self.fs,
                mu_field=mu_np, lam_field=lam_np, rho_field=rho, absorbing_frame=absorbing_frame,
                src_loc_field=src_np, wavelet_u_field=np.asarray(wavelet_u, np.float32),
                wavelet_v_field=np.asarray(wavelet_v, np.float32),
                wavelet_w_field=np.asarray(wavelet_w, np.float32), recv_loc_field=rec_np,
                isnap=isnap, surface_matrix_field=sm, num_sources=num_sources,
                num_receivers=num_receivers, device=device)
            self._fw_instance = fw
            flag = fw.run(save=True, display_callback=display_callback)
            if flag:
                print(f"Forward modeling failed with flag {flag}, reducing CFL...")
                if self._fw_instance is not None:
                    self._fw_instance.cleanup()
                    self._fw_instance = None
                continue
            print("Forward modeling completed successfully.")
            bw = BackwardModeling(
                nx=nx, nz=nz, dx=dx, dz=dz, nt=self.nt, fs=self.fs,
                mu_field=mu_np, lam_field=lam_np, rho_field=rho, absorbing_frame=absorbing_frame,
                src_loc_field=src_np, obsdata_u_field=self.observed_u,
                obsdata_v_field=self.observed_v, obsdata_w_field=self.observed_w,
                recv_loc_field=rec_np, surface_matrix_field=sm, num_sources=num_sources,
                num_receivers=num_receivers, device=device)
            self._bw_instance = bw
            flag = bw.run_calc(import_fwdata_u=fw.u_save_field, import_fwdata_v=fw.v_save_field,
                               import_fwdata_w=fw.w_save_field, isnaps_field=fw.isnaps_field,
                               num_snaps=fw.num_snaps, isnap_interval=isnap, method=method,
                               display_callback=display_callback)
            if flag:
                print(f"Backward modeling failed with flag {flag}, reducing CFL...")
                if self._bw_instance is not None:
                    self._bw_instance.cleanup()
                    self._bw_instance = None
                if self._fw_instance is not None:
                    self._fw_instance.cleanup()
                    self._fw_instance = None
                continue
            print("Backward modeling completed successfully.")
        print("\nSimulation completed.")
        print(f"Estimated velocity: {estimated_v} m/s")
        print(f"CFL: {CFL}")
        print(f"Grid: nx={nx}, nz={nz}, dx={dx:.4f}")
        self.image_u, self.image_v, self.image_w = bw.get_results()
        self.dx = dx
        self.dz = dz
        self.nx = nx
        self.nz = nz
        self.offset = 2 * absorbing_frame * dx
        self.CFL = CFL
        self.src_loc_step = src_loc_step
        return self

    def save_result(self, directory: str, savename: str):
        """rtm.py:1031-1070: same npz keys."""
        xmin = float(-self.offset)
        xmax = float(self.dx * self.nx - self.offset)
        zmin = 0.0
        zmax = float(self.dz * self.nz)
        surface_matrix = getattr(self, "surface_matrix", None)
        if not os.path.exists(directory):
            os.makedirs(directory)
        np.savez_compressed(
            os.path.join(directory, savename + ".npz"),
            u=self.image_u, v=self.image_v, w=self.image_w, receiver_loc=self.receiver_loc,
            src_loc_step=self.src_loc_step, offset=self.offset, xmin=xmin, xmax=xmax, zmin=zmin,
            zmax=zmax, dx=self.dx, dz=self.dz, nx=self.nx, nz=self.nz, surface_matrix=surface_matrix)
        print(f"Results saved to {os.path.join(directory, savename)}.npz")

    def get_results(self) -> tuple:
        return self.image_u, self.image_v, self.image_w

    def get_axes_extent(self) -> dict:
        return {"xmin": -self.offset, "xmax": self.dx * self.nx - self.offset, "zmin": 0.0,
                "zmax": self.dz * self.nz}
