"""Golden cases: systems, MCS chunks and draw seeds whose final positions were produced by the
reference updater itself (src/pscbfm/UpdaterGPUScBFM_AB_Type.cu + CRITICAL.cu, compiled for sm_100a
by oracle/Makefile) fed the engine's counter draw stream; see make_golden.py. Every case respects
the reference's limits: at most 4 bonds per monomer and int16 coordinates."""
import functools
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pscbfm_b200 import systems as S  # noqa: E402

GOLDEN_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_positions.json")

# name -> (builder, chunks of runSimulationOnGPU calls)
CASES = {
    "chains64_256x32_1000mcs": (S.small_chains, [1000]),
    "chains64_256x32_chunked": (S.small_chains, [1, 99, 400, 500]),
    "rings32_3col_2000mcs": (S.rings_and_free, [2000]),
    "sqnet64_4func_2000mcs": (S.square_network, [2000]),
    "serp32_lc16_500mcs": (lambda: S.serpentine_chains(32, 16, 0.3, seed=9), [500]),
    "serp64_lc128_300mcs": (lambda: S.serpentine_chains(64, 128, 0.4, seed=13), [300]),
    "melt256_16384x64_20mcs": (S.dense_melt, [20]),
}

# cases cheap enough for the CPU suite
FAST = [k for k in CASES if not k.startswith("melt")]


def positions_digest(xyz) -> str:
    a = np.ascontiguousarray(np.asarray(xyz, dtype="<i4").reshape(-1, 3))
    return hashlib.sha256(a.tobytes()).hexdigest()


FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_fixtures.npz")


def fixture(key: str, seed: int = 17):
    """A system converted from the reference's tests/*.bfm (make_fixtures.py)."""
    from pscbfm_b200.systems import BfmSystem, from_bonds
    z = np.load(FIXTURES)
    pairs = z[f"{key}_pairs"].astype(np.int64)
    n = z[f"{key}_xyz"].shape[0]
    # rebuild the directed lists in stored order
    cnt = np.bincount(pairs[:, 0], minlength=n).astype(np.uint32)
    maxc = max(int(cnt.max()), 1)
    ids = np.zeros((n, maxc), dtype=np.uint32)
    fill = np.zeros(n, dtype=np.int64)
    for a, b in pairs:
        ids[a, fill[a]] = b
        fill[a] += 1
    return BfmSystem(tuple(int(v) for v in z[f"{key}_box"]), z[f"{key}_xyz"].astype(np.int32), cnt, ids,
                     z[f"{key}_attributes"].astype(np.int32), z[f"{key}_forbidden"].astype(np.uint8),
                     name=key, seed=seed, periodic=tuple(bool(v) for v in z[f"{key}_periodic"]))


CASES["fixture_linearchain128_200mcs"] = (lambda: fixture("linear_chains"), [200])
FAST.append("fixture_linearchain128_200mcs")

# Boxes with walls on all three axes, pinned against the reference's NONPERIODICITY build: the
# reference's own non-periodic ring fixture (tests/Ring_N6_n6.bfm) and chains folded inside walls.
WALL_CASES = {
    "fixture_ring128_walls_3000mcs": (lambda: fixture("ring"), [3000]),
    "serp32_lc16_walls_800mcs": (lambda: S.walled(S.serpentine_chains(32, 16, 0.3, seed=21)), [300, 500]),
    "serp64_lc64_walls_300mcs": (lambda: S.walled(S.serpentine_chains(64, 64, 0.45, seed=23)), [300]),
}
CASES.update(WALL_CASES)
FAST.extend(WALL_CASES)


# The configs at their stated run lengths, pinned against the reference updater: the 256^3 melt for
# 10^4 MCS (seed 7), the 128^3 six-functional network for 10^5 MCS (seed 3; the reference's
# MAX_CONNECTIVITY 8 build) and every one of the 256 ensemble systems for 10^4 MCS alone (seeds
# 1000 + i). Generated by make_golden.py --long into reference_long.json.
LONG_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_long.json")
ENSEMBLE_MCS = 10000
LONG_CASES = {
    "melt256_16384x64_10000mcs": (S.dense_melt, [10000]),
    "network128_512x6_100000mcs": (S.crosslinked_network, [100000]),
}


@functools.lru_cache(maxsize=1)
def _ensemble():
    return tuple(S.ensemble())


def ensemble_case(i: int):
    """Member i of the 256-system ensemble (box, chain length and volume fraction drawn from the
    ensemble's generator seed; seed 1000 + i)."""
    return _ensemble()[i]


def ensemble_cases():
    return {f"ensemble256_{i:03d}_{ENSEMBLE_MCS}mcs": (lambda i=i: ensemble_case(i), [ENSEMBLE_MCS])
            for i in range(256)}
