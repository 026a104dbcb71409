"""B200-native FP64 SpGEMM engine: C = A·A and C = A·Aᵀ on CSR (int32 indices,
FP64 values), hand-written sm_100a CUDA behind a C ABI (include/spgemm_b200.h).

Host-side matrices and generators live in :mod:`appt_spgemm_b200.csr`; the
device API (``Engine``, ``run_ours``) in :mod:`appt_spgemm_b200.engine`, which
imports torch for device memory.  Importing the package loads the CUDA
library and raises if it has not been built.
"""
from . import _capi
from ._capi import SpgemmError

_capi.lib()  # fail loudly when the CUDA library is missing

__all__ = ["SpgemmError"]
