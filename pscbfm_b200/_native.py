"""Build and load the native library ``libpscbfm_b200.so`` (CUDA, sm_100a).

The library is built in-tree next to this file so that it travels with the
repository.  There is no fallback: if the shared object is missing or cannot
be loaded, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBNAME = "libpscbfm_b200.so"
LIBPATH = os.path.join(HERE, LIBNAME)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["bfm_engine.cu", "bfm_diag.cu", "bfm_color.cu", "bfm_batch.cu", "bfm_mlp.cu"]
HEADERS = ["bfm_device.cuh", "bfm_host.hpp", "bfm_sweep.cuh", "bfm_analyze.cuh", "bfm_color.hpp", "../../include/pscbfm_b200.h"]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIBPATH):
        return True
    t = os.path.getmtime(LIBPATH)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


CLI = os.path.join(HERE, "bin", "pscbfm")
CLI_SOURCES = ["pscbfm_main.cpp", "bfm_io.hpp", "../../include/UpdaterGPUScBFM_AB_Type.h"]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA sources into the in-tree shared library, and the
    pscbfm command-line simulator against it."""
    if force or _stale():
        cmd = [NVCC, *NVCC_FLAGS, "-o", LIBPATH] + [os.path.join(CSRC, s) for s in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    if force or not os.path.exists(CLI) or any(
            os.path.getmtime(os.path.join(CSRC, f)) > os.path.getmtime(CLI) for f in CLI_SOURCES) or \
            os.path.getmtime(LIBPATH) > os.path.getmtime(CLI):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"), "-I", CSRC,
               os.path.join(CSRC, "pscbfm_main.cpp"), "-o", CLI, "-L", HERE, "-lpscbfm_b200",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return LIBPATH


_lock = threading.Lock()
_lib = None

# status codes of include/pscbfm_b200.h
BFM_OK, BFM_EINVAL, BFM_ERUNTIME, BFM_ECUDA, BFM_ETIMEOUT, BFM_ENOTINIT, BFM_EUNSUPPORTED, BFM_ETOOLARGE = range(8)

_c = ctypes
_P = _c.c_void_p
_SIGS = {
    "bfm_create": (_c.c_int, [_c.POINTER(_P)]),
    "bfm_destroy": (_c.c_int, [_P]),
    "bfm_last_error": (_c.c_char_p, [_P]),
    "bfm_set_gpu": (_c.c_int, [_P, _c.c_int]),
    "bfm_copy_bond_set": (_c.c_int, [_P, _c.c_int, _c.c_int, _c.c_int, _c.c_int]),
    "bfm_set_nr_of_all_monomers": (_c.c_int, [_P, _c.c_uint32]),
    "bfm_set_attribute": (_c.c_int, [_P, _c.c_uint32, _c.c_int32]),
    "bfm_set_monomer_coordinates": (_c.c_int, [_P, _c.c_uint32, _c.c_int32, _c.c_int32, _c.c_int32]),
    "bfm_set_connectivity": (_c.c_int, [_P, _c.c_uint32, _c.c_uint32]),
    "bfm_set_lattice_size": (_c.c_int, [_P, _c.c_uint64, _c.c_uint64, _c.c_uint64]),
    "bfm_set_periodicity": (_c.c_int, [_P, _c.c_int, _c.c_int, _c.c_int]),
    "bfm_set_age": (_c.c_int, [_P, _c.c_int64]),
    "bfm_get_age": (_c.c_int, [_P, _c.POINTER(_c.c_int64)]),
    "bfm_set_rng": (_c.c_int, [_P, _c.c_int]),
    "bfm_get_rng": (_c.c_int, [_P, _c.POINTER(_c.c_int)]),
    "bfm_set_steps_between_sortings": (_c.c_int, [_P, _c.c_int64]),
    "bfm_set_all_coordinates": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_set_all_connectivity": (_c.c_int, [_P, _P, _P, _c.c_size_t]),
    "bfm_initialize": (_c.c_int, [_P]),
    "bfm_run": (_c.c_int, [_P, _c.c_uint32]),
    "bfm_get_monomer_position": (_c.c_int, [_P, _c.c_uint32, _c.POINTER(_c.c_int32), _c.POINTER(_c.c_int32), _c.POINTER(_c.c_int32)]),
    "bfm_get_positions": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_analyzer_init": (_c.c_int, [_P, _c.POINTER(_c.c_uint32)]),
    "bfm_analyze": (_c.c_int, [_P, _c.c_int, _P, _c.c_size_t]),
    "bfm_analyzer_chain_ids": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32]),
    "bfm_analyze_per_chain": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32]),
    "bfm_set_filter_stats": (_c.c_int, [_P, _c.c_int]),
    "bfm_get_filter_stats": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_cleanup": (_c.c_int, [_P]),
    "bfm_batch_create": (_c.c_int, [_c.c_int, _c.POINTER(_P)]),
    "bfm_batch_destroy": (_c.c_int, [_P]),
    "bfm_batch_last_error": (_c.c_char_p, [_P]),
    "bfm_batch_add_system": (_c.c_int, [_P, _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.c_uint32, _P, _P, _P, _P, _c.c_int,
                                         _c.c_int64, _c.c_int64, _P, _c.c_uint64, _P]),
    "bfm_batch_initialize": (_c.c_int, [_P]),
    "bfm_batch_set_clusters": (_c.c_int, [_P, _c.c_int]),
    "bfm_batch_set_autotune": (_c.c_int, [_P, _c.c_int]),
    "bfm_batch_get_clusters": (_c.c_int, [_P, _P, _P, _P]),
    "bfm_batch_run": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_batch_get_positions": (_c.c_int, [_P, _c.c_uint32, _P, _c.c_size_t]),
    "bfm_batch_get_state": (_c.c_int, [_P, _c.c_uint32, _P, _P, _P]),
    "bfm_batch_get_all_positions": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_batch_gather_positions": (_c.c_int, [_P, _P, _c.c_size_t, _P]),
    "bfm_batch_get_lattice": (_c.c_int, [_P, _c.c_uint32, _P, _c.c_size_t, _P]),
    "bfm_batch_info": (_c.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "bfm_set_sweep_autotune": (_c.c_int, [_P, _c.c_int]),
    "bfm_get_sweep_tuning": (_c.c_int, [_P, _P, _P, _P, _P, _P, _P, _c.c_uint32]),
    "bfm_batch_set_shape": (_c.c_int, [_P, _c.c_int, _c.c_int]),
    "bfm_batch_get_tuning": (_c.c_int, [_P, _P, _P, _P, _P, _P]),
    "bfm_mlp_create": (_c.c_int, [_c.c_int, _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.c_uint64, _c.POINTER(_P)]),
    "bfm_mlp_destroy": (_c.c_int, [_P]),
    "bfm_mlp_last_error": (_c.c_char_p, [_P]),
    "bfm_mlp_num_params": (_c.c_int, [_P, _P]),
    "bfm_mlp_set_params": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_mlp_get_params": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_mlp_forward": (_c.c_int, [_P, _P, _c.c_uint32, _P]),
    "bfm_mlp_gradients": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32, _P, _c.c_size_t, _P]),
    "bfm_mlp_train_step": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32, _c.c_float, _P]),
    "bfm_mlp_train_steps": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32, _P, _P, _c.c_uint32, _c.c_float, _P]),
    "bfm_mlp_last_ms": (_c.c_int, [_P, _P]),
    "bfm_get_lattice": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_get_lattice_words": (_c.c_int, [_P, _c.POINTER(_c.c_size_t)]),
    "bfm_get_nspecies": (_c.c_int, [_P, _c.POINTER(_c.c_uint32)]),
    "bfm_get_colors": (_c.c_int, [_P, _P, _c.c_size_t]),
    "bfm_get_species_order": (_c.c_int, [_P, _c.c_uint32, _P, _c.c_size_t, _c.POINTER(_c.c_size_t)]),
    "bfm_get_counters": (_c.c_int, [_P, _P]),
    "bfm_get_last_run_ms": (_c.c_int, [_P, _c.POINTER(_c.c_double)]),
    "bfm_get_last_run_launches": (_c.c_int, [_P, _c.POINTER(_c.c_uint64)]),
    "bfm_set_launch_mode": (_c.c_int, [_P, _c.c_int]),
    "bfm_time_kernels": (_c.c_int, [_P, _c.c_uint32, _c.POINTER(_c.c_double), _c.POINTER(_c.c_uint64), _c.POINTER(_c.c_uint64)]),
    "bfm_set_barrier_timeout_ms": (_c.c_int, [_P, _c.c_uint32]),
    "bfm_set_sweep_shape": (_c.c_int, [_P, _c.c_int]),
    "bfm_get_launch_info": (_c.c_int, [_P, _c.POINTER(_c.c_int), _c.POINTER(_c.c_int), _c.POINTER(_c.c_int),
                                       _c.POINTER(_c.c_size_t)]),
    "bfm_barrier_selftest": (_c.c_int, [_c.c_int, _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.POINTER(_c.c_double)]),
    "bfm_barrier_selftest_variant": (_c.c_int, [_c.c_int, _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.c_int, _c.c_uint32,
                                                _c.POINTER(_c.c_double)]),
    "bfm_color_graph": (_c.c_int, [_c.c_uint32, _P, _P, _c.c_int, _P, _P]),
    "bfm_color_graph_device": (_c.c_int, [_c.c_int, _c.c_uint32, _P, _P, _c.c_int, _P, _P, _P]),
    "bfm_set_coloring": (_c.c_int, [_P, _c.c_int]),
    "bfm_get_coloring": (_c.c_int, [_P, _P, _P]),
    "bfm_substep_noalloc": (_c.c_int, [_P, _P, _P, _P, _c.c_uint32, _P, _c.c_uint32, _c.c_uint32, _c.c_uint32, _P,
                                       _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.c_uint32, _c.c_int, _P]),
    "bfm_debug_philox_vs_curand": (_c.c_int, [_c.c_int, _c.c_uint64, _c.c_uint64, _c.c_uint64, _c.c_uint32, _P]),
    "bfm_r250_seed": (_c.c_int, [_c.c_uint64]),
    "bfm_r250_seed_words": (_c.c_int, [_P, _c.c_size_t]),
    "bfm_r250_get_state": (_c.c_int, [_P]),
    "bfm_r250_set_state": (_c.c_int, [_P]),
    "bfm_r250_rand32": (_c.c_uint32, []),
}


def exported_symbols() -> list[str]:
    """Names of every entry point declared in include/pscbfm_b200.h."""
    return list(_SIGS)


def lib() -> ctypes.CDLL:
    """Load the native library (building it first if the sources are newer)."""
    global _lib
    with _lock:
        if _lib is None:
            if _stale():
                build()
            if not os.path.exists(LIBPATH):
                raise RuntimeError(f"{LIBPATH} is missing: build the CUDA extension first")
            L = ctypes.CDLL(LIBPATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib
