"""Build librtm_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m taichirtm_b200.build
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "librtm_b200.so")
# bounds-checking build (every kernel access checked against the call's buffers)
DEBUG_LIB = os.path.join(LIBDIR, "librtm_b200_debug.so")
SOURCES = ["rtm_api.cu", "noalloc.cu"]
DEPS = ["plan_host.h", "ckpt_pack.cuh", "step_kernels.cuh", "step2_kernels.cuh", "checkpoint_kernels.cuh", "debug_bounds.cuh", "aux_kernels.cuh", "adjoint_kernels.cuh", "adjoint2_kernels.cuh", "noalloc.cu"]
# -fmad=false: no FMA contraction, so every cell's FP32 arithmetic follows the
# reference's expression order exactly and results do not depend on the launch
# shape the autotuner picks (the kernels are HBM-bound; FLOPs are free).
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def _stale(out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    files = [os.path.join(CSRC, f) for f in SOURCES + DEPS]
    files.append(os.path.join(HERE, "..", "include", "rtm_b200.h"))
    return any(os.path.exists(f) and os.path.getmtime(f) > t for f in files)


def build(force=False, verbose=False, debug=False):
    """Build librtm_b200.so, or with debug=True the bounds-checking
    librtm_b200_debug.so (-DRTM_BOUNDS_CHECK).  Returns the library path."""
    out = DEBUG_LIB if debug else LIB
    if not force and not _stale(out):
        return out
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    srcs = [os.path.join(CSRC, f) for f in SOURCES if os.path.exists(os.path.join(CSRC, f))]
    cmd = [nvcc, *NVCC_FLAGS, *(["-DRTM_BOUNDS_CHECK"] if debug else []), *srcs, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed building {os.path.basename(out)}")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, debug="--debug" in sys.argv))
