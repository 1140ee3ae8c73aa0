"""fvmhd3d_b200: B200-native (sm_100a) fluid hot path of the moving-mesh MHD
code fvmhd3d, behind a C-ABI that mirrors the reference's `system` call
sequence.  See include/fvmhd3d_b200.h for the native interface."""
from .mesh import Mesh, build_periodic, jittered_lattice  # noqa: F401
from .system import System, FvmError, FVM_PREC_FP64, FVM_PREC_FP32  # noqa: F401
from .ordering import sort_local_data, hilbert_keys  # noqa: F401
from . import problems  # noqa: F401

__all__ = ["Mesh", "build_periodic", "jittered_lattice", "System", "FvmError", "problems",
           "FVM_PREC_FP64", "FVM_PREC_FP32", "sort_local_data", "hilbert_keys"]
