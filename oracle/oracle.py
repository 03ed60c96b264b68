"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes bindings of the CPU restatement of the reference sweep (oracle/bfm_oracle.cpp, built as
oracle/liboracle.so) and of the reference updater compiled for sm_100a
(oracle/_ref/libpscbfm_ref*.so, GPU only). Only tests/, the smoke entry and the baseline legs of
bench.py (CPU baseline, reference arm) import this module; the engine in pscbfm_b200/ never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libpscbfm_ref.so")
REF_LIB_NP = os.path.join(HERE, "_ref", "libpscbfm_ref_np.so")
REF_LIB_C8 = os.path.join(HERE, "_ref", "libpscbfm_ref_c8.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")

_lib = None
_ref = {}


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_hash.argtypes = [C.c_uint32]
        L.orc_hash.restype = C.c_uint32
        L.orc_counter_draw.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_counter_draw.restype = C.c_uint32
        L.orc_counter_draws.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u32p]
        L.orc_counter_draws.restype = None
        L.orc_bond_index.argtypes = [C.c_int32] * 3
        L.orc_bond_index.restype = C.c_uint32
        L.orc_color.argtypes = [C.c_uint32, _u32p, _u32p, C.c_uint32, _u8p, C.c_char_p, C.c_int]
        L.orc_color.restype = C.c_int
        L.orc_run.argtypes = [C.c_uint32, _i32p, _u32p, _u32p, C.c_uint32, _u32p, C.c_uint32, _u8p, C.c_int,
                              C.c_uint64, C.c_uint64, _u32p, C.c_uint64, C.c_uint32, _i32p, _u64p,
                              C.c_char_p, C.c_int]
        L.orc_run.restype = C.c_int
        L.orc_seq_run.argtypes = [C.c_uint32, _i32p, _u32p, _u32p, C.c_uint32, _u32p, C.c_uint32, _u8p, C.c_uint64,
                                  C.c_uint32, _i32p, _u64p, C.c_char_p, C.c_int]
        L.orc_seq_run.restype = C.c_int
        _lib = L
    return _lib


def _arrs(sys):
    xyz = np.ascontiguousarray(sys.xyz, dtype=np.int32).reshape(-1)
    cnt = np.ascontiguousarray(sys.nbr_count, dtype=np.uint32)
    ids = np.ascontiguousarray(sys.nbr_ids, dtype=np.uint32).reshape(-1)
    box = np.ascontiguousarray(sys.box, dtype=np.uint32)
    forb = np.ascontiguousarray(sys.forbidden, dtype=np.uint8)
    return xyz, cnt, ids, box, forb


def move_hash(a: int) -> int:
    return int(lib().orc_hash(a))


def counter_draws(seed: int, k0: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint32)
    lib().orc_counter_draws(seed, k0, count, out)
    return out


def color(sys) -> np.ndarray:
    xyz, cnt, ids, box, forb = _arrs(sys)
    out = np.zeros(sys.n, dtype=np.uint8)
    err = C.create_string_buffer(512)
    nc = lib().orc_color(sys.n, cnt, ids, sys.maxc, out, err, 512)
    if nc < 0:
        raise RuntimeError(err.value.decode())
    return out


def run(sys, n_mcs: int, seed: int | None = None, substep0: int = 0, draws=None):
    """Positions after n_mcs MCS of the parallel sweep, plus (attempted, tentative, accepted)."""
    xyz, cnt, ids, box, forb = _arrs(sys)
    out = np.zeros_like(xyz)
    stats = np.zeros(3, dtype=np.uint64)
    err = C.create_string_buffer(512)
    if draws is None:
        kind, dl = 0, np.zeros(1, np.uint32)
        seed = sys.seed if seed is None else seed
    else:
        kind, dl = 1, np.ascontiguousarray(draws, dtype=np.uint32)
        seed = 0
    rc = lib().orc_run(sys.n, xyz, cnt, ids, sys.maxc, box, sys.walls, forb, kind, seed, substep0, dl,
                       len(dl), n_mcs, out, stats, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out.reshape(-1, 3), tuple(int(s) for s in stats)


def seq_run(sys, n_mcs: int, seed: int):
    xyz, cnt, ids, box, forb = _arrs(sys)
    out = np.zeros_like(xyz)
    stats = np.zeros(2, dtype=np.uint64)
    err = C.create_string_buffer(512)
    rc = lib().orc_seq_run(sys.n, xyz, cnt, ids, sys.maxc, box, sys.walls, forb, seed, n_mcs, out, stats, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out.reshape(-1, 3), tuple(int(s) for s in stats)


# ------------------------------------------------------------------ reference updater (on a GPU)

def _ref_path(walls: int, conn: int = 0) -> str:
    """The default build for periodic boxes, the NONPERIODICITY build for boxes with walls on all
    three axes (the reference has no build for mixed periodicity), the MAX_CONNECTIVITY 8 build for
    periodic systems with more than 4 bonds on some monomer (the reference has no build with both)."""
    if conn > 8:
        raise ValueError("the reference updater accepts at most 8 bonds per monomer")
    if walls == 0:
        return REF_LIB if conn <= 4 else REF_LIB_C8
    if walls == 7 and conn <= 4:
        return REF_LIB_NP
    raise ValueError("the reference updater supports fully periodic boxes, or fully non-periodic ones with at "
                     "most 4 bonds per monomer")


def _conn(sys) -> int:
    return int(np.max(sys.nbr_count)) if sys.n else 0


def ref_available(walls: int = 0, conn: int = 0) -> bool:
    return os.path.exists(_ref_path(walls, conn))


def ref_lib(walls: int = 0, conn: int = 0):
    path = _ref_path(walls, conn)
    if path not in _ref:
        R = C.CDLL(path)
        R.bfmref_run.argtypes = [C.c_int, C.c_uint32, _i32p, _u32p, _u32p, C.c_uint32, _u32p, _u8p,
                                 _u32p, C.c_uint64, _u32p, C.c_uint32, _i32p, _u64p, C.c_char_p, C.c_int]
        R.bfmref_run.restype = C.c_int
        R.bfmref_time.argtypes = [C.c_int, C.c_uint32, _i32p, _u32p, _u32p, C.c_uint32, _u32p, _u8p,
                                  _u32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.POINTER(C.c_float), C.POINTER(C.c_double), _i32p, C.c_char_p, C.c_int]
        R.bfmref_time.restype = C.c_int
        R.bfmref_max_connectivity.argtypes = []
        R.bfmref_max_connectivity.restype = C.c_int
        _ref[path] = R
    return _ref[path]


def ref_run(sys, draws, chunks, gpu: int = 0):
    """Runs the reference updater (its own kernels; the NONPERIODICITY build for a box with walls,
    the MAX_CONNECTIVITY 8 build for more than 4 bonds per monomer) with the given draw list; chunks
    are the nMCS of successive runSimulationOnGPU calls. Returns positions and the number of draws
    used."""
    xyz, cnt, ids, box, forb = _arrs(sys)
    out = np.zeros_like(xyz)
    used = np.zeros(1, dtype=np.uint64)
    err = C.create_string_buffer(1024)
    d = np.ascontiguousarray(draws, dtype=np.uint32)
    ch = np.ascontiguousarray(chunks, dtype=np.uint32)
    rc = ref_lib(sys.walls, _conn(sys)).bfmref_run(gpu, sys.n, xyz, cnt, ids, sys.maxc, box, forb, d, len(d), ch,
                                                   len(ch), out, used, err, 1024)
    if rc != 0:
        raise RuntimeError(f"reference updater failed ({rc}): {err.value.decode()}")
    return out.reshape(-1, 3), int(used[0])


def ref_time(sys, warm_mcs: int, timed_mcs: int, reps: int = 1, gpu: int = 0):
    """Times the reference updater on the system with the counter draw stream of its seed: one
    untimed runSimulationOnGPU(warm_mcs), then `reps` timed calls of timed_mcs MCS. Returns
    (device ms, host seconds, final positions), sums over the timed calls; every call includes the
    reference's own copy-back of the positions."""
    xyz, cnt, ids, box, forb = _arrs(sys)
    n_colors = int(color(sys).max()) + 1 if sys.n else 1
    draws = counter_draws(sys.seed, 0, 2 * n_colors * (warm_mcs + reps * timed_mcs))
    out = np.zeros_like(xyz)
    ms = C.c_float(0.0)
    wall = C.c_double(0.0)
    err = C.create_string_buffer(1024)
    rc = ref_lib(sys.walls, _conn(sys)).bfmref_time(gpu, sys.n, xyz, cnt, ids, sys.maxc, box, forb, draws,
                                                    len(draws), warm_mcs, timed_mcs, reps, C.byref(ms),
                                                    C.byref(wall), out, err, 1024)
    if rc != 0:
        raise RuntimeError(f"reference updater failed ({rc}): {err.value.decode()}")
    return float(ms.value), float(wall.value), out.reshape(-1, 3)


# ------------------------------------------------------------------ observables (int64 recomputation)

def molecules(sys):
    """Connected components of the bond graph, numbered by their lowest monomer id."""
    parent = list(range(sys.n))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a
    rows, cols = sys.bonds()
    for a, b in zip(rows.tolist(), cols.tolist()):
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    roots = np.array([find(i) for i in range(sys.n)])
    _, first_idx, mol = np.unique(roots, return_index=True, return_inverse=True)
    # np.unique sorts by root id = lowest member id, which is the required numbering
    return mol.astype(np.int64)


def observables(sys, xyz, xyz_ref):
    """The int64 words of bfm_observables, recomputed from positions with numpy (exact int64)."""
    xyz = np.asarray(xyz, dtype=np.int64)
    ref = np.asarray(xyz_ref, dtype=np.int64)
    mol = molecules(sys)
    m = int(mol.max()) + 1
    out = np.zeros(5 * m + 513, dtype=np.int64)
    mom = np.zeros((m, 4), dtype=np.int64)
    for a in range(3):
        np.add.at(mom[:, a], mol, xyz[:, a])
    np.add.at(mom[:, 3], mol, (xyz ** 2).sum(axis=1))
    out[:4 * m] = mom.reshape(-1)
    idx = np.arange(sys.n)
    first = np.full(m, sys.n, dtype=np.int64)
    last = np.full(m, -1, dtype=np.int64)
    np.minimum.at(first, mol, idx)
    np.maximum.at(last, mol, idx)
    d = xyz[last] - xyz[first]
    out[4 * m:5 * m] = (d ** 2).sum(axis=1)
    rows, cols = sys.bonds()
    bi = (xyz[cols] - xyz[rows]) & 7
    code = bi[:, 0] | (bi[:, 1] << 3) | (bi[:, 2] << 6)
    out[5 * m:5 * m + 512] = np.bincount(code, minlength=512)
    out[5 * m + 512] = ((xyz - ref) ** 2).sum()
    return out
