"""Test-only checkers for the MPM substep (never part of the product path).

* ``oracle.cpu``   -- ctypes wrapper of liboracle.so, the FP64 CPU restatement
                      of the reference substep (mpm_oracle.c).
* ``oracle.ref``   -- ctypes wrapper of _ref/libmpm_ref.so, the reference's
                      own MPMCUDA.cu built unmodified for sm_100a behind a
                      headless harness (needs a GPU to run).
* ``oracle.numpy_mpm`` -- an independent NumPy restatement of the substep
                      (2D Taichi scripts and the 3D CUDA kernels), used to
                      cross-check the C oracle.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.
"""
