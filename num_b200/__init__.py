"""num_b200 -- B200-native (sm_100a) sparse hot path: CSR SpMV, multi-RHS and
many-matrix SpMV, CG with its vector ops, halo pack/unpack.

`num_b200.kokkos_spmv` is the drop-in for the reference's `kokkos_spmv` module;
the C ABI is include/num_b200.h (libnum_b200.so, loaded by num_b200._lib).
"""
from . import generators  # noqa: F401

__version__ = "0.1.0"
