"""tmd_b200 -- Python host side of the B200 pair_style tensormd force path.

The compute path is libtmd_b200.so (CUDA, sm_100a) behind the C ABI of
include/tmd_b200.h; this package only binds it with ctypes and mirrors the
LAMMPS-facing interface of PairTensorMD (src/ML-TENSORMD/pair_tensormd.cpp).
There is no CPU fallback: importing a class that needs the library raises if
libtmd_b200.so is missing or cannot find a CUDA device.
"""
from .lib import TmdError, library_path, load_library
from .pair import (PairTensorMD, TensorMDBatch, TensorMDModel, TensorMDServer,
                   TensorMDSystem)

__all__ = ["TmdError", "library_path", "load_library", "PairTensorMD",
           "TensorMDBatch", "TensorMDModel", "TensorMDServer", "TensorMDSystem"]
