"""kettle_b200 — B200-native circuit propagation behind kettle's API.

The engine is the CUDA library libkettle_b200.so (C-ABI in
include/kettle_b200.h); `capi` binds it from Python, `workloads` builds seeded
circuits and Hamiltonians, `autograd` wraps the adjoint gradient as a
torch.autograd.Function.  The C++20 drop-in front end (namespace `ket`) lives
in include/kettle/ and kettle_b200/host/.
"""
from . import capi, workloads  # noqa: F401
from .capi import (KT_APPLY_FUSED, KT_APPLY_PER_GATE, KT_C64, KT_C128, DensityMatrix,  # noqa: F401
                   KettleError, Statevector)

__all__ = ["capi", "workloads", "Statevector", "DensityMatrix", "KettleError", "KT_C128", "KT_C64",
           "KT_APPLY_FUSED", "KT_APPLY_PER_GATE"]
