"""Parity of the CUDA engine (through the C-ABI) with the reference and the oracle: bit-exact
final positions, for every engine path, at the configs' sizes and on ragged / odd cases."""
import json

import numpy as np
import pytest

import pscbfm_b200 as P
from cases import CASES, GOLDEN_JSON, positions_digest
from oracle import oracle as O
from pscbfm_b200 import systems as S

pytestmark = pytest.mark.gpu

MODES = {"launch": P.MODE_LAUNCH, "graph": P.MODE_GRAPH, "resident": P.MODE_RESIDENT, "auto": P.MODE_AUTO,
         "persistent": P.MODE_PERSISTENT, "cluster": P.MODE_CLUSTER}
REPRS = {"codes": P.REPR_AUTO, "gather": P.REPR_GATHER}


def run_engine(s, chunks, mode=P.MODE_AUTO, seed=None, repr_=P.REPR_AUTO):
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, seed=seed, mode=mode, representation=repr_)
    if repr_ == P.REPR_AUTO:
        assert u.representation() != 0, "symmetric systems with <= 6 bonds use bond codes"
    for c in chunks:
        u.runSimulationOnGPU(c)
    xyz = u.get_coords().copy()
    st = u.stats()
    u.validate()
    u.close()
    return xyz, st


def _resident_ok(s):
    return max(s.box) <= 64


@pytest.mark.parametrize("repr_", ["codes", "gather"])
@pytest.mark.parametrize("mode", ["launch", "graph", "resident", "persistent", "cluster"])
@pytest.mark.parametrize("name", list(CASES))
def test_engine_reproduces_reference_updater(name, mode, repr_):
    g = json.load(open(GOLDEN_JSON))["cases"][name]
    build, chunks = CASES[name]
    s = build()
    if mode == "resident" and not _resident_ok(s):
        pytest.skip("box larger than the resident kernel holds")
    xyz, st = run_engine(s, chunks, MODES[mode], repr_=REPRS[repr_])
    assert positions_digest(xyz) == g["sha256"]
    assert st["mcs"] == sum(chunks)


NON_CUBIC = {
    "serp64x32x128_lc32": (lambda: S.serpentine_chains((64, 32, 128), 32, 0.4, seed=31), [150, 50]),
    "serp16x64x32_lc16_walls_xz": (lambda: S.walled(S.serpentine_chains((16, 64, 32), 16, 0.35, seed=33), walls=5),
                                   [200]),
    "serp128x8x16_lc8": (lambda: S.serpentine_chains((128, 8, 16), 8, 0.3, seed=35), [300]),
    "serp8x8x256_lc32": (lambda: S.serpentine_chains((8, 8, 256), 32, 0.3, seed=37), [120, 180]),
    # walled axes whose sides are not powers of two (the lattice side is the next power of two)
    "serp48x40x24_lc16_walls_xyz": (lambda: S.walled(S.serpentine_chains((48, 40, 24), 16, 0.35, seed=43), walls=7),
                                    [200]),
    "serp36x64x32_lc16_walls_x": (lambda: S.walled(S.serpentine_chains((36, 64, 32), 16, 0.35, seed=45), walls=1),
                                  [150, 50]),
    "serp64x32x100_lc32_walls_z": (lambda: S.walled(S.serpentine_chains((64, 32, 100), 32, 0.3, seed=47), walls=4),
                                   [120]),
}


@pytest.mark.parametrize("repr_", ["codes", "gather"])
@pytest.mark.parametrize("mode", ["launch", "graph", "resident", "persistent", "cluster"])
@pytest.mark.parametrize("name", list(NON_CUBIC))
def test_non_cubic_boxes_vs_oracle(name, mode, repr_):
    """Boxes with unequal sides (powers of two, or any side >= 4 along a walled axis): the brick
    index interleaves the axes' low bits and appends the longer axes' high bits. The reference updater always indexes its lattice by an
    interleaved Z-curve, which runs past its lattice array when the sides differ, so the oracle
    (a linear lattice) alone pins these. The resident mode falls back to the graph path where a
    system does not fit one CTA."""
    build, chunks = NON_CUBIC[name]
    s = build()
    want, _ = O.run(s, sum(chunks))
    xyz, st = run_engine(s, chunks, MODES[mode], repr_=REPRS[repr_])
    assert np.array_equal(xyz, want)
    assert st["mcs"] == sum(chunks)


@pytest.mark.parametrize("build", [S.crosslinked_network, lambda: S.serpentine_chains(128, 64, 0.3, seed=3),
                                   lambda: S.serpentine_chains(64, 64, 0.8, seed=13),
                                   lambda: S.walled(S.serpentine_chains((128, 32, 64), 16, 0.35, seed=41), walls=6)])
def test_cluster_kernel_vs_oracle(build):
    """Systems too large for one CTA's shared memory, held by a cluster of CTAs: the cluster path
    runs (bfm_get_path) and every chunk of the run equals the oracle."""
    s = build()
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, mode=P.MODE_CLUSTER)
    assert u.path() == P.MODE_CLUSTER, s.name
    done = 0
    for chunk in (1, 9, 40):
        u.runSimulationOnGPU(chunk)
        done += chunk
        want, ost = O.run(s, done)
        assert np.array_equal(u.get_coords(), want), (s.name, done)
    u.validate()
    st = u.stats()
    assert st["mcs"] == done and (st["attempted"], st["tentative"], st["accepted"]) == ost
    u.close()


def test_asymmetric_lists_fall_back_to_gather():
    # a bond listed in one direction only: the reference checks it from one side only
    xyz = np.array([[2 * j, 0, 0] for j in range(16)])
    s = S.from_bonds((32, 32, 32), xyz, [(j, j + 1) for j in range(15)], seed=8)
    s.nbr_count = s.nbr_count.copy()
    s.nbr_count[5] = 1       # monomer 5 forgets its second neighbour (6); 6 still lists 5
    ref, _ = O.run(s, 150)
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    assert u.representation() == 0
    u.runSimulationOnGPU(150)
    assert np.array_equal(u.get_coords(), ref)
    u.close()


def test_engine_matches_live_reference_updater():
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    s = S.small_chains()
    draws = O.counter_draws(s.seed, 0, 2 * 2 * 300)
    ref, used = O.ref_run(s, draws, [100, 200])
    assert used == len(draws)
    xyz, _ = run_engine(s, [300])
    assert np.array_equal(xyz, ref)


@pytest.mark.parametrize("repr_", ["codes", "gather"])
@pytest.mark.parametrize("mode", ["launch", "graph"])
def test_six_functional_network_vs_oracle(mode, repr_):
    # the reference is compiled with MAX_CONNECTIVITY 4, so this case is pinned by the oracle only
    s = S.crosslinked_network()
    ref, ost = O.run(s, 1000)
    xyz, st = run_engine(s, [400, 600], MODES[mode], repr_=REPRS[repr_])
    assert np.array_equal(xyz, ref)
    assert (st["attempted"], st["tentative"], st["accepted"]) == ost


@pytest.mark.parametrize("repr_", ["codes", "gather"])
@pytest.mark.parametrize("mode", ["launch", "graph", "resident", "persistent", "cluster"])
@pytest.mark.parametrize("walls", [1, 4, 6])
def test_partial_walls_vs_oracle(walls, mode, repr_):
    # the reference has builds for fully periodic and fully walled boxes only: mixed periodicity
    # is pinned by the oracle
    s = S.walled(S.serpentine_chains(32, 32, 0.35, seed=31), walls=walls)
    ref, ost = O.run(s, 400)
    xyz, st = run_engine(s, [150, 250], MODES[mode], repr_=REPRS[repr_])
    assert np.array_equal(xyz, ref)
    assert (st["attempted"], st["tentative"], st["accepted"]) == ost


@pytest.mark.parametrize("mode", ["launch", "graph", "resident", "persistent", "cluster"])
def test_hydrogel_fixture_with_walls_vs_oracle(mode):
    # the reference's non-periodic hydrogel (tests/coloring-test-Hydrogel...bfm): up to 5 bonds per
    # monomer, more than the reference build's MAX_CONNECTIVITY, so the oracle pins it
    from cases import fixture
    s = fixture("hydrogel")
    ref, ost = O.run(s, 600)
    xyz, st = run_engine(s, [600], MODES[mode])
    assert np.array_equal(xyz, ref)
    assert (st["attempted"], st["tentative"], st["accepted"]) == ost


def test_dense_melt_full_config():
    """256^3 melt at phi = 0.5: the full 10^4 MCS of the config, split across calls and modes,
    equals one uninterrupted run; invariants hold; the first MCS match the oracle."""
    s = S.dense_melt()
    ref, _ = O.run(s, 4)
    xyz4, _ = run_engine(s, [4], P.MODE_GRAPH)
    assert np.array_equal(xyz4, ref)
    a, sa = run_engine(s, [10000], P.MODE_GRAPH)
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, mode=P.MODE_LAUNCH)
    u.runSimulationOnGPU(3000)
    u.set_mode(P.MODE_GRAPH)
    u.runSimulationOnGPU(7000)
    b = u.get_coords().copy()
    u.validate()
    u.close()
    assert np.array_equal(a, b)
    assert sa["attempted"] == 10000 * s.n


def test_mode_switches_mid_run():
    s = S.serpentine_chains(64, 32, 0.35, seed=21)
    ref, _ = O.run(s, 150)
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, mode=P.MODE_LAUNCH)
    u.runSimulationOnGPU(30)
    u.set_mode(P.MODE_RESIDENT)
    u.runSimulationOnGPU(30)
    u.set_mode(P.MODE_GRAPH)
    u.runSimulationOnGPU(30)
    u.set_mode(P.MODE_PERSISTENT)
    u.runSimulationOnGPU(30)
    u.set_mode(P.MODE_LAUNCH)
    u.runSimulationOnGPU(30)
    assert np.array_equal(u.get_coords(), ref)
    u.close()


def test_callback_stream_equals_counter_stream():
    s = S.rings_and_free()
    k = iter(range(10 ** 9))
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    u.set_draw_callback(lambda: P.updater.counter_draw(s.seed, next(k)))
    u.runSimulationOnGPU(200)
    xyz = u.get_coords().copy()
    u.close()
    ref, _ = O.run(s, 200)
    assert np.array_equal(xyz, ref)


def test_set_coords_after_initialize():
    s = S.small_chains()
    mid, _ = O.run(s, 25)
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    u.runSimulationOnGPU(10)
    u.set_coords(mid)   # replaces the state; the draw stream continues at sub-step 20
    u.runSimulationOnGPU(15)
    got = u.get_coords().copy()
    u.close()
    s2 = S.BfmSystem(s.box, mid.astype(np.int32), s.nbr_count, s.nbr_ids, s.attributes, s.forbidden, seed=s.seed)
    ref, _ = O.run(s2, 15, substep0=20)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("resident,cluster", [(True, True), (False, True), (True, False)])
def test_batch_equals_each_system_alone(resident, cluster):
    systems = S.ensemble(n_systems=20)
    systems.append(S.rings_and_free())         # three colours in the mix
    systems.append(S.crosslinked_network())    # 64-bit bond codes in the mix
    systems.append(S.walled(S.serpentine_chains(64, 32, 0.3, seed=41)))   # walls in the mix
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    # and two systems forced onto the gather representation
    for s in systems[:2]:
        members.append(P.UpdaterGPUScBFM_AB_Type(0).load_system(s, representation=P.REPR_GATHER))
    systems = systems + systems[:2]
    b = P.Batch(members, resident=resident, cluster=cluster)
    b.run(60)
    b.run(40)
    for s, m in zip(systems, members):
        ref, _ = O.run(s, 100)
        assert np.array_equal(m.get_coords(), ref), s.name
        m.validate()
    b.close()
    for m in members:
        m.close()


def test_batch_autotune_keeps_trajectories():
    """The autotuner's trials are ordinary MCS under different paths, kernel shapes and CTA sizes:
    every member ends where the oracle puts it after the same number of MCS."""
    systems = S.ensemble(n_systems=10, base_seed=700) + [S.crosslinked_network(), S.rings_and_free()]
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members)
    rep = b.autotune(3)
    # stage 1: the paths (the network runs in a cluster of CTAs alone, so the cluster path is a
    # dimension); stage 2: the grid check's register budget x CTA size for the best paths (the
    # 128^3 members run on the grid-phase kernels under every path choice); stage 3: the perform's
    # warps per CTA x per tile for the best of those
    paths, grid, perf = rep["trials"][:4], rep["trials"][4:16], rep["trials"][16:]
    assert {(t["resident"], t["cluster"]) for t in paths} == {(r, c) for r in (True, False) for c in (True, False)}
    assert {(t["shape"], t["block"]) for t in grid} == {(s, bl) for s in range(4) for bl in (128, 256, 512)}
    assert all(t["perform"] == (0, 0) for t in paths + grid)
    assert [t["perform"] for t in perf] == [(8, 4), (4, 2), (8, 8), (2, 2)]
    assert len({(t["shape"], t["block"]) for t in perf}) == 1
    assert len(rep["trials"]) == 20 and rep["mcs_spent"] == 20 * 4
    best = min(rep["trials"], key=lambda t: t["ms_per_mcs"])
    assert rep["perform"] == best["perform"] and b.perform_shape() == best["perform"]
    assert rep["ms_per_mcs"] == min(t["ms_per_mcs"] for t in rep["trials"])
    b.run(17)
    for s, m in zip(systems, members):
        ref, _ = O.run(s, rep["mcs_spent"] + 17)
        assert np.array_equal(m.get_coords(), ref), s.name
        m.validate()
    b.close()
    for m in members:
        m.close()


@pytest.mark.parametrize("cluster", [True, False])
def test_batch_cluster_members_vs_oracle(cluster):
    """Members too large for one CTA that a cluster of CTAs holds run in the cluster-resident kernel
    inside a batch (one launch per run and cluster size, entries strided by the member count),
    beside resident and grid-phase members, with uneven MCS per member: every trajectory equals the
    oracle's."""
    systems = [S.crosslinked_network(), S.serpentine_chains(64, 64, 0.8, seed=13), S.small_chains(),
               S.serpentine_chains(128, 64, 0.3, seed=3), S.serpentine_chains(128, 32, 0.1, seed=17)]
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members, cluster=cluster)
    plan = [[40, 7, 25, 3, 0], [0, 33, 25, 12, 41]]
    for mcs in plan:
        b.run_each(mcs)
    totals = np.sum(plan, axis=0)
    for s, m, t in zip(systems, members, totals):
        ref, _ = O.run(s, int(t))
        assert np.array_equal(m.get_coords(), ref), s.name
        assert m.stats()["mcs"] == t
        m.validate()
    b.close()
    # the two cluster members alone: one launch per cluster size and run, not two per sub-step
    pair = P.Batch(members[:2], cluster=cluster)
    n0 = pair.launch_count()
    pair.run(5)
    launched = pair.launch_count() - n0
    if cluster:
        assert launched <= 2
    else:
        assert launched >= 2 * 5 * 2   # a check and a perform per sub-step, two colours or more
    pair.close()
    for s, m, t in zip(systems[:2], members[:2], totals[:2]):
        ref, _ = O.run(s, int(t) + 5)
        assert np.array_equal(m.get_coords(), ref), s.name
    for m in members:
        m.close()


def test_sharded_batch_runner_on_one_gpu():
    """run_sharded on one rank with the Batch runner: each system's positions and MCS count equal
    running it alone (the multi-rank assignment and gather are tested over gloo on the CPU)."""
    from pscbfm_b200 import sharding
    systems = [S.serpentine_chains(32, 16, 0.3, seed=81), S.crosslinked_network(),
               S.walled(S.serpentine_chains((48, 40, 24), 16, 0.35, seed=43), walls=7)]
    mcs = [30, 12, 20]
    res = sharding.run_sharded(systems, mcs, sharding.batch_runner(0))
    for s, m, (xyz, st) in zip(systems, mcs, res):
        want, _ = O.run(s, m)
        assert np.array_equal(xyz, want), s.name
        assert st["mcs"] == m


@pytest.mark.parametrize("resident", [True, False])
def test_batch_uneven_mcs_per_member(resident):
    """run_each: members advance different MCS counts (some idle) in one launch sequence, as the
    server runs them; each trajectory stays its own."""
    systems = S.ensemble(n_systems=8, base_seed=300) + [S.rings_and_free()]
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members, resident=resident)
    plan = [[37, 0, 100, 1, 64, 65, 3, 0, 29], [5, 80, 0, 99, 1, 0, 70, 12, 29]]
    for mcs in plan:
        b.run_each(mcs)
    totals = np.sum(plan, axis=0)
    for s, m, t in zip(systems, members, totals):
        ref, _ = O.run(s, int(t))
        assert np.array_equal(m.get_coords(), ref), s.name
        assert m.stats()["mcs"] == t
        m.validate()
    b.close()
    for m in members:
        m.close()


def test_single_monomer_and_ragged_groups():
    # one free monomer, and a 33-monomer chain (groups of 17 and 16: ragged tiles)
    one = S.from_bonds((8, 8, 8), np.array([[1, 1, 1]]), np.zeros((0, 2)), seed=4)
    xyz = np.array([[2 * j, 0, 0] for j in range(33)])
    chain = S.from_bonds((128, 128, 128), xyz, [(j, j + 1) for j in range(32)], seed=5)
    for s in (one, chain):
        for mode in ("launch", "graph", "resident"):
            ref, _ = O.run(s, 120)
            got, _ = run_engine(s, [120], MODES[mode])
            assert np.array_equal(got, ref), (s.name, mode)


def test_batch_lone_grid_members_vs_oracle():
    """A grid group with a single system runs the single-system kernels inside the batch: the
    network (bond codes) and an asymmetric chain (gather representation), each alone in its group
    beside resident systems, for enough sub-steps that the batch's captured graph runs too; every
    member equals the oracle."""
    net = S.crosslinked_network()
    xyz = np.array([[2 * j, 0, 0] for j in range(16)])
    asym = S.from_bonds((128, 128, 128), xyz, [(j, j + 1) for j in range(15)], seed=8)
    asym.nbr_count = asym.nbr_count.copy()
    asym.nbr_count[5] = 1
    small = [S.serpentine_chains(32, 16, 0.3, seed=40 + i) for i in range(3)]
    systems = [net, asym] + small
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members)
    b.run(70)
    for s, m in zip(systems, members):
        want, _ = O.run(s, 70)
        assert np.array_equal(m.get_coords(), want), s.name
        m.validate()
    for m in members:
        m.close()


@pytest.mark.parametrize("block", [128, 256, 512])
@pytest.mark.parametrize("name", ["melt256_16384x64_20mcs", "serp64_lc128_300mcs", "chains64_256x32_chunked"])
def test_check_block_sizes_vs_reference(name, block):
    """The bond-code check with 128, 256 or 512 threads over the same 512-monomer tile (4, 2 or 1
    monomers per thread), on the graph path and one launch at a time: identical to the reference."""
    g = json.load(open(GOLDEN_JSON))["cases"][name]
    build, chunks = CASES[name]
    s = build()
    for mode in (P.MODE_GRAPH, P.MODE_LAUNCH):
        u = P.UpdaterGPUScBFM_AB_Type(0)
        u.load_system(s, mode=mode)
        u.set_grid_block(block)
        for c in chunks:
            u.runSimulationOnGPU(c)
        assert positions_digest(u.get_coords()) == g["sha256"], (name, block, mode)
        u.close()


def test_check_block_size_rejects_other_sizes():
    u = P.UpdaterGPUScBFM_AB_Type(0)
    with pytest.raises(ValueError, match="128, 256 or 512"):
        u.set_grid_block(64)
    u.close()


@pytest.mark.parametrize("warps,group", [(1, 1), (2, 2), (4, 2), (8, 4), (8, 8), (4, 1)])
@pytest.mark.parametrize("name", ["melt256_16384x64_20mcs", "chains64_256x32_chunked"])
def test_perform_shapes_vs_reference(name, warps, group):
    """The bond-code perform with 1 to 8 warps per CTA and per tile, on the graph path and one
    launch at a time: identical to the reference."""
    g = json.load(open(GOLDEN_JSON))["cases"][name]
    build, chunks = CASES[name]
    s = build()
    for mode in (P.MODE_GRAPH, P.MODE_LAUNCH):
        u = P.UpdaterGPUScBFM_AB_Type(0)
        u.load_system(s, mode=mode)
        u.set_perform(warps, group)
        for c in chunks:
            u.runSimulationOnGPU(c)
        assert positions_digest(u.get_coords()) == g["sha256"], (warps, group, mode)
        u.close()


def test_perform_shape_rejects_other_shapes():
    u = P.UpdaterGPUScBFM_AB_Type(0)
    for w, g in [(3, 1), (4, 8), (0, 4), (16, 16)]:
        with pytest.raises(ValueError, match="1, 2, 4 or 8"):
            u.set_perform(w, g)
    u.close()
