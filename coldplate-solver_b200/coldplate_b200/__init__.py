"""B200-native SIMPLE solver for cold-plate flow (drop-in for the reference's
2-D staggered-grid SIMPLE iteration).  The compute path is libcoldplate.so:
hand-written sm_100a CUDA kernels behind the C ABI in include/cp_simple.h."""
from . import cases
from ._native import CpError, PREC_FP64, PREC_MIXED, default_params, lib
from .solver import Batch, Simple, make_params, partition_fields
from .thermal import Thermal

__all__ = ["Simple", "Batch", "partition_fields", "Thermal", "make_params", "cases", "CpError", "PREC_FP64", "PREC_MIXED", "default_params", "lib"]
