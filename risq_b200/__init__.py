"""risq_b200: the HCI variational hot path of RISQ on one B200.

Sparse Hamiltonian construction over a determinant set, sigma = H v, and the
Davidson eigensolver, in hand-written sm_100a CUDA behind the C ABI of
include/risqgpu.h (librisqgpu.so, built in this directory).
"""
from . import _capi
from .fcidump import Integrals, read_fcidump, synthetic_integrals, write_fcidump
from .gpu import DavidsonResult, GpuHam, device_count

__all__ = ["GpuHam", "DavidsonResult", "Integrals", "read_fcidump", "write_fcidump", "synthetic_integrals",
           "device_count", "_capi"]
