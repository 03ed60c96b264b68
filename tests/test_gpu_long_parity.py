"""The configs at their stated run lengths, bit-exact against the reference updater itself.

The hashes in tests/golden/reference_long.json were produced by the reference's own GPU updater
(src/pscbfm, compiled for sm_100a by oracle/Makefile; the six-functional network by its
MAX_CONNECTIVITY 8 build) fed the engine's counter draw stream (make_golden.py --long):
  - the 256^3 melt, 1,048,576 monomers, 10^4 MCS, seed 7;
  - the 128^3 six-functional network, 11,264 monomers, 10^5 MCS, seed 3;
  - each of the 256 ensemble systems run alone for 10^4 MCS, seeds 1000 + i.
The engine reproduces them on its single-system paths and as one 256-member Batch."""
import json
import os

import numpy as np
import pytest

import pscbfm_b200 as P
from cases import LONG_CASES, LONG_JSON, ENSEMBLE_MCS, ensemble_case, ensemble_cases, positions_digest

pytestmark = pytest.mark.gpu


def golden(name):
    if not os.path.exists(LONG_JSON):
        pytest.fail("tests/golden/reference_long.json is missing (make_golden.py --long)")
    return json.load(open(LONG_JSON))["cases"][name]


def run_engine(s, chunks, mode, repr_=P.REPR_AUTO):
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, mode=mode, representation=repr_)
    for c in chunks:
        u.runSimulationOnGPU(c)
    xyz = u.get_coords().copy()
    st = u.stats()
    u.validate()
    u.close()
    return xyz, st


@pytest.mark.parametrize("mode,repr_,chunks", [
    (P.MODE_AUTO, P.REPR_AUTO, [10000]),
    (P.MODE_LAUNCH, P.REPR_AUTO, [1, 2999, 7000]),
    (P.MODE_PERSISTENT, P.REPR_AUTO, [10000]),
    (P.MODE_GRAPH, P.REPR_GATHER, [5000, 5000]),
])
def test_dense_melt_10k_mcs_vs_reference(mode, repr_, chunks):
    name = "melt256_16384x64_10000mcs"
    g = golden(name)
    build, ref_chunks = LONG_CASES[name]
    s = build()
    assert sum(chunks) == sum(ref_chunks) == 10000
    xyz, st = run_engine(s, chunks, mode, repr_)
    assert positions_digest(xyz) == g["sha256"]
    assert st["attempted"] == 10000 * s.n


@pytest.mark.parametrize("mode,repr_,chunks", [
    (P.MODE_AUTO, P.REPR_AUTO, [100000]),
    (P.MODE_GRAPH, P.REPR_AUTO, [30000, 70000]),
    (P.MODE_PERSISTENT, P.REPR_AUTO, [100000]),
    (P.MODE_GRAPH, P.REPR_GATHER, [100000]),
])
def test_network_100k_mcs_vs_reference(mode, repr_, chunks):
    name = "network128_512x6_100000mcs"
    g = golden(name)
    build, _ = LONG_CASES[name]
    s = build()
    xyz, st = run_engine(s, chunks, mode, repr_)
    assert positions_digest(xyz) == g["sha256"]
    u = P.UpdaterGPUScBFM_AB_Type(0).load_system(s)
    assert u.n_colors()[0] == g["n_colors"]
    u.close()


def test_ensemble_256_batch_10k_mcs_vs_reference():
    """All 256 ensemble systems in one Batch, tuned on the run's first MCS, for 10^4 MCS: every
    member equals the reference updater run on that system alone."""
    names = list(ensemble_cases())
    gold = [golden(nm) for nm in names]
    systems = [ensemble_case(i) for i in range(256)]
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members)
    b.run(3)
    tuned = b.autotune(2)
    done = 3 + tuned["mcs_spent"]              # the trials advance every member
    assert all(m.stats()["mcs"] == done for m in members)
    b.run(ENSEMBLE_MCS - done)
    b.synchronize()
    bad = [nm for nm, m, g in zip(names, members, gold) if positions_digest(m.get_coords()) != g["sha256"]]
    for m in members:
        m.validate()
    b.close()
    for m in members:
        m.close()
    assert not bad, f"{len(bad)} of 256 members differ from the reference, first {bad[:4]}"


@pytest.mark.parametrize("i", [0, 17, 101, 255])
def test_ensemble_member_alone_vs_reference(i):
    """A few ensemble members on the single-system default path (AUTO picks resident, cluster,
    persistent or graph by size)."""
    name = list(ensemble_cases())[i]
    g = golden(name)
    xyz, _ = run_engine(ensemble_case(i), [ENSEMBLE_MCS], P.MODE_AUTO)
    assert positions_digest(xyz) == g["sha256"]
