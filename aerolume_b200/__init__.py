"""B200-native incompressible Navier-Stokes step for Aerolume's ns2d / ns3d solvers.

Hand-written sm_100a CUDA kernels behind a C ABI (``include/aero_b200.h``), loaded with
ctypes from the in-tree ``libaero_b200.so``.  There is no CPU fallback: every compute
call raises ``RuntimeError`` when the library or a CUDA device is missing.
"""
__version__ = "0.1.0"
