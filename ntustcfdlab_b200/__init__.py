"""B200 implementation of NTUSTCFD's projection-method time step.

The compute path is ``lib/libntcfd.so`` (CUDA kernels for sm_100a behind the
C-ABI of ``include/ntcfd.h``); ``solver`` drives it from Python with the
reference's initialisation and step sequence, ``cases`` holds the measured
workloads.  There is no CPU fallback: loading fails when the library is
missing.
"""
__all__ = ["abi", "solver", "cases", "build"]
