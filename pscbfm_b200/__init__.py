"""B200-native colored bond-fluctuation-model sweep (drop-in for the hot path
of lgh0504/pscbfm's UpdaterGPUScBFM_AB_Type).

The compute path is the CUDA library ``libpscbfm_b200.so`` (sm_100a) behind
the C ABI in ``include/pscbfm_b200.h``; this package holds the ctypes
bindings, a host-side mirror of the reference's updater class and the
synthetic system generators.
"""
from . import systems  # noqa: F401
from ._native import build, lib  # noqa: F401
from .updater import (  # noqa: F401
    CudaError,
    DeviceTimeout,
    Rng,
    UpdaterGPUScBFM_AB_Type,
    color_graph,
    r250_get_state,
    r250_rand32,
    r250_seed,
    r250_seed_words,
    r250_set_state,
)
from .batch import Batch, BatchError  # noqa: F401,E402
