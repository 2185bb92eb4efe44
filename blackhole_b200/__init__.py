"""B200-native Kerr null-geodesic tracer (sm_100a CUDA behind a C ABI).

Submodules: ``kerr`` (host API), ``_abi`` (ctypes mirror of include/bh_kerr.h),
``build`` (in-tree build of the CUDA library).
"""
__all__ = ["kerr"]
