"""ctypes binding of libbfm.so (include/bfm.h). There is no fallback: if the CUDA library is
missing or the machine has no GPU, the calls fail loudly."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbfm.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "bfm.h")

BFM_OK = 0
BFM_ERR_INVALID_ARGUMENT = 1
BFM_ERR_RUNTIME = 2
BFM_ERR_CUDA = 3
BFM_ERR_OUT_OF_RANGE = 4
BFM_ERR_NULL_HANDLE = 5
BFM_ERR_BUDGET = 6
BFM_ERR_BUSY = 7

MODE_AUTO, MODE_LAUNCH, MODE_GRAPH, MODE_RESIDENT, MODE_PERSISTENT, MODE_CLUSTER = 0, 1, 2, 3, 4, 5

DRAW_FN = C.CFUNCTYPE(C.c_uint32, C.c_void_p)


class BfmCudaError(RuntimeError):
    """A CUDA runtime error inside the engine (the reference would exit the process)."""


class BfmBudgetError(RuntimeError):
    """A server job does not fit the memory budget."""


class BfmBusy(RuntimeError):
    """A server result is not ready yet."""


class NoallocSystem(C.Structure):
    """bfm_noalloc_system of include/bfm.h."""
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("nbr", C.c_void_p), ("nnb", C.c_void_p),
                ("npad", C.c_uint32), ("maxc", C.c_uint32), ("box", C.c_uint32 * 3), ("n_colors", C.c_uint32),
                ("group_offset", C.c_void_p), ("group_size", C.c_void_p), ("forbidden", C.c_void_p)]


_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

H = C.c_void_p

# name -> (argtypes); every function returns int status unless listed in _RET
_SIGS = {
    "bfm_create": [C.POINTER(C.c_void_p), C.c_int],
    "bfm_destroy": [H],
    "bfm_set_gpu": [H, C.c_int],
    "bfm_cleanup": [H],
    "bfm_set_periodicity": [H, C.c_int, C.c_int, C.c_int],
    "bfm_set_n_monomers": [H, C.c_uint32],
    "bfm_set_attribute": [H, C.c_uint32, C.c_int32],
    "bfm_set_coords": [H, C.c_uint32, C.c_int32, C.c_int32, C.c_int32],
    "bfm_set_coords_bulk": [H, _i32p, C.c_uint32],
    "bfm_add_bond": [H, C.c_uint32, C.c_uint32],
    "bfm_add_bonds_bulk": [H, _u32p, C.c_uint32],
    "bfm_set_attributes_bulk": [H, _i32p, C.c_uint32],
    "bfm_set_box": [H, C.c_uint32, C.c_uint32, C.c_uint32],
    "bfm_set_bond_forbidden": [H, C.c_int, C.c_int, C.c_int, C.c_int],
    "bfm_set_standard_bond_set": [H],
    "bfm_populate_lattice": [H],
    "bfm_set_seed": [H, C.c_uint64],
    "bfm_set_draw_callback": [H, DRAW_FN, C.c_void_p],
    "bfm_set_substep": [H, C.c_uint64],
    "bfm_get_substep": [H, C.POINTER(C.c_uint64)],
    "bfm_set_mode": [H, C.c_int],
    "bfm_set_representation": [H, C.c_int],
    "bfm_get_representation": [H, C.POINTER(C.c_int)],
    "bfm_batch_launch_count": [H, C.POINTER(C.c_uint64)],
    "bfm_initialize": [H],
    "bfm_run": [H, C.c_int32],
    "bfm_run_async": [H, C.c_int32],
    "bfm_synchronize": [H],
    "bfm_inject_barrier_stall": [H],
    "bfm_get_path": [H, C.POINTER(C.c_int)],
    "bfm_get_coord": [H, C.c_uint32, C.c_int, C.POINTER(C.c_int32)],
    "bfm_get_coords_bulk": [H, _i32p, C.c_uint32],
    "bfm_n_colors": [H, C.POINTER(C.c_uint32), C.c_void_p, C.c_uint32],
    "bfm_get_stats": [H, C.POINTER(C.c_uint64)],   # a ctypes buffer: read once per step by callers
    "bfm_stats_enqueue": [H, C.POINTER(C.c_uint64)],
    "bfm_stats_wait": [H, C.c_uint64, C.POINTER(C.c_uint64)],
    "bfm_validate": [H],
    "bfm_device_bytes": [H, C.POINTER(C.c_uint64)],
    "bfm_run_timed": [H, C.c_int32, C.POINTER(C.c_float)],
    "bfm_n_molecules": [H, C.POINTER(C.c_uint32)],
    "bfm_molecule_sizes": [H, _u32p, C.c_uint32],
    "bfm_observables": [H, _i64p, C.c_uint64],
    "bfm_reset_msd_reference": [H],
    "bfm_time_kernels": [H, C.c_int32, _f64p],
    "bfm_launch_count": [H, C.POINTER(C.c_uint64)],
    "bfm_transfer_bytes": [H, C.POINTER(C.c_uint64)],
    "bfm_probe_device": [C.c_int, _f64p],
    "bfm_batch_create": [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p), C.c_uint32],
    "bfm_batch_destroy": [H],
    "bfm_batch_run": [H, C.c_int32],
    "bfm_batch_run_async": [H, C.c_int32],
    "bfm_batch_run_each": [H, _i32p],
    "bfm_batch_set_shape": [H, C.c_int],
    "bfm_batch_set_block": [H, C.c_int],
    "bfm_batch_set_perform": [H, C.c_int, C.c_int],
    "bfm_batch_get_perform": [H, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "bfm_set_grid_block": [H, C.c_int],
    "bfm_set_perform": [H, C.c_int, C.c_int],
    "bfm_batch_autotune": [H, C.c_int32, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float),
                           np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_uint32,
                           C.POINTER(C.c_uint32)],
    "bfm_batch_run_timed": [H, C.c_int32, C.POINTER(C.c_float)],
    "bfm_batch_synchronize": [H],
    "bfm_batch_set_resident": [H, C.c_int],
    "bfm_batch_set_cluster": [H, C.c_int],
    "bfm_sweep_noalloc": [C.c_void_p, C.c_int32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_char_p, C.c_size_t],
    "bfm_server_create": [C.POINTER(C.c_void_p), C.c_int, C.c_uint64, C.c_uint32],
    "bfm_server_destroy": [H],
    "bfm_server_submit": [H, H, C.c_int32, C.c_int32, C.POINTER(C.c_uint64)],
    "bfm_server_estimate_bytes": [H, C.POINTER(C.c_uint64)],
    "bfm_server_status": [H, C.c_uint64, C.POINTER(C.c_int)],
    "bfm_server_cancel": [H, C.c_uint64],
    "bfm_server_wait": [H, C.c_uint64, C.c_double],
    "bfm_server_result": [H, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32),
                          C.POINTER(C.c_double)],
    "bfm_server_stats": [H, _f64p],
    "bfm_server_job_times": [H, C.c_uint64, _f64p],
    "bfm_server_sample_words": [H, C.c_uint64, C.POINTER(C.c_uint64)],
    "bfm_server_inject_fault": [H, C.c_int],
    "bfm_color_graph": [C.c_uint32, _u32p, _u32p, C.c_uint32,
                        np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"), C.POINTER(C.c_uint32)],
}
_RET = {"bfm_last_error": C.c_char_p, "bfm_batch_last_error": C.c_char_p, "bfm_counter_draw": C.c_uint32,
        "bfm_server_last_error": C.c_char_p}
_RET_ARGS = {"bfm_last_error": [H], "bfm_batch_last_error": [H], "bfm_counter_draw": [C.c_uint64, C.c_uint64],
             "bfm_server_last_error": [H]}

_lib = None


def declared_symbols() -> list[str]:
    """Every function name include/bfm.h declares."""
    import re
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(bfm_\w+)\s*\(", txt, re.M)))


def load():
    """Loads libbfm.so and declares every signature. Raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python pscbfm_b200/build.py` "
                          "(the engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    for name, rt in _RET.items():
        f = getattr(L, name)
        f.argtypes = _RET_ARGS[name]
        f.restype = rt
    _lib = L
    return L


def raise_for(status: int, msg: str):
    if status == BFM_OK:
        return
    if status == BFM_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == BFM_ERR_OUT_OF_RANGE:
        raise IndexError(msg)
    if status == BFM_ERR_CUDA:
        raise BfmCudaError(msg)
    if status == BFM_ERR_BUDGET:
        raise BfmBudgetError(msg)
    if status == BFM_ERR_BUSY:
        raise BfmBusy(msg)
    raise RuntimeError(msg)
