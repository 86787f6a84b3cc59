"""Imaging utilities with the reference's interface (src/imaging.py).

``stack_rtm_images`` performs the cross-shot sum on the GPU in FP64 (the
reference sums on the host at the inputs' dtype, imaging.py:81-93) and returns
float32 like the reference.  The display helpers are host NumPy, as in the
reference."""
import glob
import os
from typing import Any, Dict, List, Optional

import numpy as np
import torch


def load_rtm_results(directory: str, pattern: str = "*.npz") -> List[Dict[str, Any]]:
    """Load every npz written by ReverseTimeMigration.save_result
    (imaging.py:29-54); each dict also carries its 'filepath'."""
    results = []
    for path in glob.glob(os.path.join(directory, pattern)):
        with np.load(path, allow_pickle=True) as data:
            entry = {k: data[k] for k in data.files}
        entry["filepath"] = path
        results.append(entry)
    return results


def _sum_fp64(arrays):
    """FP64 sum of the per-shot images on the GPU.  There is no host path:
    without a visible CUDA device this raises."""
    from .plan import require_cuda
    require_cuda()
    acc = None
    for a in arrays:
        t = torch.as_tensor(np.asarray(a)).to("cuda", torch.float64)
        acc = t if acc is None else acc + t
    return acc.cpu().numpy()


def stack_rtm_images(results: List[Dict[str, Any]], subtract_mean: bool = True) -> Dict[str, np.ndarray]:
    """Sum the u, v, w images of all results, transpose to (nz, nx), optionally
    remove the mean, and attach the extent of the last result
    (imaging.py:57-129)."""
    if not results:
        raise ValueError("No results to stack")
    out = {}
    for c in ("u", "v", "w"):
        dtype = np.asarray(results[0][c]).dtype
        img = _sum_fp64([r[c] for r in results]).astype(dtype).T
        if subtract_mean:
            img = img - np.mean(img)
        out[c] = img
    last = results[-1]
    offset, dx, dz = float(last["offset"]), float(last["dx"]), float(last["dz"])
    nx, nz = int(last["nx"]), int(last["nz"])
    xmin, xmax, zmin, zmax = -offset, dx * nx - offset, 0.0, dz * nz
    out.update(xmin=xmin, xmax=xmax, zmin=zmin, zmax=zmax, extent=[xmin, xmax, zmax, zmin],
               dx=dx, dz=dz, nx=nx, nz=nz)
    return out


def compute_display_limits(data: np.ndarray) -> tuple:
    """Symmetric limits (-max|data|, max|data|) (imaging.py:132-147)."""
    m = np.max(np.abs(data))
    return -m, m


def prepare_image_data(image: np.ndarray, attenuate_region: Optional[tuple] = None,
                       attenuation_factor: float = 1e-3) -> np.ndarray:
    """Copy of ``image`` with a clipped (x0, x1, z0, z1) box scaled by
    ``attenuation_factor`` (imaging.py:150-182)."""
    result = image.copy()
    if attenuate_region is not None:
        x0, x1, z0, z1 = attenuate_region
        x0, z0 = max(0, x0), max(0, z0)
        x1, z1 = min(result.shape[0], x1), min(result.shape[1], z1)
        if x0 < x1 and z0 < z1:
            result[x0:x1, z0:z1] *= attenuation_factor
    return result


def create_visualization_data(rtm_instance, subtract_mean: bool = True, attenuate_source: bool = True,
                              source_attenuation_radius: int = 10) -> Dict[str, Any]:
    """Display-ready images of one ReverseTimeMigration (imaging.py:185-248):
    optional damping around the source (1e-3 on u/w in a box, 1e-1 on v over
    the source rows), transpose, optional mean removal, limits."""
    u = rtm_instance.image_u.copy()
    v = rtm_instance.image_v.copy()
    w = rtm_instance.image_w.copy()
    if attenuate_source and hasattr(rtm_instance, "src_loc_step"):
        si, sj = rtm_instance.src_loc_step[0]
        r = source_attenuation_radius
        x0, x1 = max(0, si - r), min(u.shape[0], si + r)
        z0, z1 = sj, min(u.shape[1], sj + r)
        u[x0:x1, z0:z1] *= 1e-3
        v[:, z0:z1] *= 1e-1
        w[x0:x1, z0:z1] *= 1e-3
    maps = [u.T, v.T, w.T]
    if subtract_mean:
        maps = [m - np.mean(m) for m in maps]
    e = rtm_instance.get_axes_extent()
    out = dict(u=maps[0], v=maps[1], w=maps[2], xmin=e["xmin"], xmax=e["xmax"], zmin=e["zmin"],
               zmax=e["zmax"], extent=[e["xmin"], e["xmax"], e["zmax"], e["zmin"]])
    out.update(u_lim=compute_display_limits(maps[0]), v_lim=compute_display_limits(maps[1]),
               w_lim=compute_display_limits(maps[2]))
    return out


def save_stacked_results(data: Dict[str, Any], filepath: str):
    """npz with u, v, w and the extent (imaging.py:251-277)."""
    d = os.path.dirname(filepath)
    if d and not os.path.exists(d):
        os.makedirs(d)
    np.savez_compressed(filepath, u=data["u"], v=data["v"], w=data["w"], xmin=data["xmin"],
                        xmax=data["xmax"], zmin=data["zmin"], zmax=data["zmax"])
    print(f"Stacked results saved to {filepath}")
