"""B200 implementation of the Axilrod-Teller three-body hot path of ThreeBodyMDAlgorithms
(NATA / AUTA / P3BCA forces and the Simulation step), behind the C ABI in include/tbmd.h.

The compute path is libtbmd.so (hand-written sm_100a CUDA kernels); importing a submodule that
needs it raises if the library has not been built (python -m threebodymdalgorithms_b200.build).
"""
from ._lib import AUTA, FP64, MIXED, NATA, P3BCA, Context, TbmdError, load, rank_layout  # noqa: F401

__all__ = ["Context", "TbmdError", "load", "rank_layout", "NATA", "AUTA", "P3BCA", "FP64", "MIXED"]
