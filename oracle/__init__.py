"""CPU restatements of TaichiRTM's elastic RTM hot path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package, and only as the checker or the timed
CPU baseline.  The product (``taichirtm_b200``) never calls into it: its GPU
path fails loudly when the CUDA library is missing.

Contents
  fd_oracle.py  vectorised NumPy restatement (FP64 or FP32) of
                src/forward_modeling.py and src/backward_modeling.py and of the
                rtm.py helpers the path needs.  Pinned against golden vectors
                recorded from the unmodified reference source
                (tests/golden/make_golden.py).
  rtm_oracle.c  the same per-step sequence in C/OpenMP, compiled for float
                and double; the timed CPU baseline and the checker at sizes
                NumPy is too slow for.
  c_oracle.py   ctypes wrapper of the compiled C restatement.
"""
