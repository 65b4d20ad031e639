"""B200-native searchlight alignment backend for the hyperalignment C API.

The compute path is ``libha_b200.so`` (hand-written sm_100a CUDA behind a C
ABI, include/hyperalignment_b200.h); this package holds its ctypes binding
(``_lib``), the reference-shaped Python wrapper (``hyperalignment_c``), the
device-resident plan (``plan``), the learned (alpha, PC count) proposal
(``learned``), one hemisphere sharded over several GPUs (``shard``) and the
synthetic workload generators (``workloads``).
"""

from . import _lib  # noqa: F401
from .hyperalignment_c import (  # noqa: F401
    cleanup,
    searchlight_procrustes,
    searchlight_procrustes_csc,
    searchlight_ridge_csc,
    searchlight_weights,
    sparse_pattern,
)
