"""A NumPy-backed stand-in for the small part of the Taichi API that the
reference modules use, so that ``src/forward_modeling.py``,
``src/backward_modeling.py`` and ``src/rtm.py`` of TaichiRTM can be imported
and run UNMODIFIED, serially, in FP64, on tiny grids.

Test infrastructure only: it is used by ``make_golden.py`` to record golden
input/output vectors from the reference's own code; nothing in the product
imports it.

Why serial execution reproduces the reference's parallel semantics: every
reference kernel is Jacobi-style -- it reads only fields it does not write in
the same loop (forward_modeling.py:330-347, 367-384; backward_modeling.py:
331-345, 365-380) -- so any iteration order gives the same values.  The only
order-dependent case is the atomic ``+=`` of several sources on one cell
(forward_modeling.py:432-443), which the serial loop performs in source order.

Limitation: ``ti.atomic_max(result, k)`` on a kernel-local scalar
(forward_modeling.py:474-488) cannot mutate a Python local, so
``_check_finite`` always returns 0 here.  Failure codes are pinned by the
restatement's own tests instead.

Numbers: f32 fields are held as float64 NumPy arrays, so the run is an FP64
execution of the reference's arithmetic (IEEE semantics, including 1/0 = inf
on the edge cells of ``inv_rho_u``/``inv_rho_w``).
"""
import itertools
import types

import numpy as np

f32 = "f32"
f64 = "f64"
i32 = "i32"

cpu = "cpu"
gpu = "gpu"
cuda = "cuda"
vulkan = "vulkan"
opengl = "opengl"
metal = "metal"


class _Field:
    def __init__(self, dtype, shape):
        if isinstance(shape, int):
            shape = (shape,)
        self.shape = tuple(int(s) for s in shape)
        self.dtype = dtype
        npdt = np.int64 if dtype == i32 else np.float64
        self.data = np.zeros(self.shape, dtype=npdt)

    def __getitem__(self, idx):
        return self.data[idx]

    def __setitem__(self, idx, val):
        self.data[idx] = val

    def __iter__(self):
        if len(self.shape) == 1:
            return iter(range(self.shape[0]))
        return itertools.product(*[range(s) for s in self.shape])

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        assert arr.shape == self.shape, (arr.shape, self.shape)
        self.data[...] = arr

    def to_numpy(self):
        return self.data.copy()


def field(dtype, shape):
    return _Field(dtype, shape)


def data_oriented(cls):
    return cls


def kernel(fn):
    def run(*args, **kwargs):
        with np.errstate(all="ignore"):
            return fn(*args, **kwargs)
    run.__name__ = fn.__name__
    run.__doc__ = fn.__doc__
    return run


def template():
    return "template"


def static(x):
    return x


def loop_config(**kwargs):
    return None


def block_local(*args):
    return None


def ndrange(*dims):
    ranges = []
    for d in dims:
        if isinstance(d, (tuple, list)):
            ranges.append(range(int(d[0]), int(d[1])))
        else:
            ranges.append(range(int(d)))
    return itertools.product(*ranges)


def exp(x):
    return np.exp(x)


def abs(x):  # noqa: A001 - mirrors ti.abs
    return np.abs(x)


def atomic_max(a, b):
    return max(a, b)


def init(**kwargs):
    return None


def reset():
    return None


def as_module():
    mod = types.ModuleType("taichi")
    for name, val in dict(globals()).items():
        if not name.startswith("__") and name not in ("itertools", "types", "np", "as_module"):
            setattr(mod, name, val)
    return mod
