"""Error behaviour of the drop-in API mirrors the reference's exceptions
(src/pscbfm/UpdaterGPUScBFM_AB_Type.cu: invalid_argument / runtime_error / out_of_range)."""
import pytest

import pscbfm_b200 as P
from pscbfm_b200 import systems as S

pytestmark = pytest.mark.gpu


def fresh():
    return P.UpdaterGPUScBFM_AB_Type(0)


def test_set_gpu_out_of_range():
    u = fresh()
    with pytest.raises(ValueError, match="not present"):
        u.setGpu(999)


def test_monomer_outside_walls_rejected():
    from pscbfm_b200 import systems as S
    s = S.walled(S.serpentine_chains(32, 16, 0.3, seed=5), walls=2)
    s.xyz = s.xyz.copy()
    s.xyz[0, 1] = 31          # corner at L-1 along the walled axis: the cube would stick out
    u = fresh()
    with pytest.raises(RuntimeError, match="outside the walls"):
        u.load_system(s)
    u.close()
    s.xyz[0, 1] = 30          # at L-2 it fits
    v = fresh().load_system(s)
    with pytest.raises(ValueError, match="outside the walls"):
        bad = v.get_coords().copy()
        bad[5, 1] = -1
        v.set_coords(bad)
    v.close()


def test_periodicity_fixed_after_initialize():
    from pscbfm_b200 import systems as S
    u = fresh().load_system(S.small_chains())
    with pytest.raises(RuntimeError, match="before initialize"):
        u.setPeriodicity(False, False, False)
    u.close()


def test_monomer_count_set_twice():
    u = fresh()
    u.setNrOfAllMonomers(4)
    with pytest.raises(RuntimeError, match="already set"):
        u.setNrOfAllMonomers(5)


def test_box_must_be_power_of_two():
    with pytest.raises(RuntimeError, match="power of 2"):
        fresh().setLatticeSize(48, 64, 64)
    with pytest.raises(ValueError):
        fresh().setLatticeSize(2048, 64, 64)


def test_walled_axis_of_any_side():
    """A walled axis takes any side >= 4; a periodic one needs a power of two, whichever of
    setPeriodicity and setLatticeSize comes first."""
    u = fresh()
    u.setPeriodicity(False, True, True)
    u.setLatticeSize(48, 64, 64)
    with pytest.raises(RuntimeError, match="power of 2"):
        u.setPeriodicity(True, True, True)
    v = fresh()
    v.setPeriodicity(False, False, True)
    with pytest.raises(RuntimeError, match="power of 2"):
        v.setLatticeSize(48, 40, 24)
    v.setLatticeSize(48, 40, 32)
    with pytest.raises(RuntimeError, match="power of 2"):
        v.setLatticeSize(48, 40, 3)


def test_too_many_bonds():
    u = fresh()
    u.setNrOfAllMonomers(20)
    for j in range(1, 17):
        u.setConnectivity(0, j)
    with pytest.raises(ValueError, match="maximum amount of bonds"):
        u.setConnectivity(0, 17)


def test_index_errors():
    u = fresh()
    u.setNrOfAllMonomers(3)
    with pytest.raises(IndexError):
        u.setMonomerCoordinates(3, 0, 0, 0)
    with pytest.raises(IndexError):
        u.setConnectivity(0, 7)


def test_wrong_bond_set_and_double_initialize():
    s = S.small_chains()
    u = fresh()
    u.load_system(s, initialize=False)
    u.copyBondSet(3, 1, 0, True)
    with pytest.raises(RuntimeError, match="Expected 108 allowed bonds, but got 107"):
        u.initialize()
    u.copyBondSet(3, 1, 0, False)
    u.initialize()
    with pytest.raises(RuntimeError, match="Initialize was already called"):
        u.initialize()


def test_run_before_initialize():
    u = fresh()
    u.setNrOfAllMonomers(2)
    with pytest.raises(RuntimeError, match="initialize"):
        u.runSimulationOnGPU(1)


def test_cleanup_allows_repeat():
    s = S.small_chains()
    u = fresh()
    u.load_system(s)
    u.runSimulationOnGPU(5)
    a = u.get_coords().copy()
    u.cleanup()
    u.load_system(s)
    u.runSimulationOnGPU(5)
    assert (u.get_coords() == a).all()


def test_reference_getters_and_colours():
    s = S.rings_and_free()
    u = fresh()
    u.load_system(s)
    assert u.getMonomerPositionInX(0) == s.xyz[0, 0]
    assert u.getMonomerPositionInY(1) == s.xyz[1, 1]
    assert u.getMonomerPositionInZ(2) == s.xyz[2, 2]
    n, sizes = u.n_colors()
    assert n == 3 and sizes.sum() == s.n
    assert u.execute() is True
    assert u.device_bytes() > 0


def test_lemonade_adapter_runs_like_the_oracle(tmp_path):
    """The LeMonADE-style program of tests/lemonade_stub/caller.cpp (two bonded monomers in a 32^3
    box, the 108-vector set, 100 MCS of the counter stream with seed 7) ends where the oracle does,
    and the adapter advances the molecules' age."""
    import os
    import subprocess
    import numpy as np
    from oracle import oracle as O
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    exe = tmp_path / "lemonade_caller"
    r = subprocess.run(["g++", "-std=c++14", "-I", os.path.join(root, "include"),
                        "-I", os.path.join(here, "lemonade_stub"), os.path.join(here, "lemonade_stub", "caller.cpp"),
                        "-o", str(exe), "-L", os.path.join(root, "pscbfm_b200"), "-lbfm",
                        "-Wl,-rpath," + os.path.join(root, "pscbfm_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    lines = run.stdout.split("\n")
    got = np.array([[int(v) for v in ln.split()] for ln in lines[:2]])
    assert lines[2] == "age 100"
    s = S.from_bonds((32, 32, 32), np.array([[0, 0, 0], [2, 0, 0]]), [(0, 1)], seed=7)
    ref, _ = O.run(s, 100)
    assert np.array_equal(got, ref)


def _adapter_input(s, steps, calls):
    lines = [f"box {s.box[0]} {s.box[1]} {s.box[2]}", "periodic " + " ".join(str(int(p)) for p in s.periodic),
             f"monomers {s.n}"]
    lines += [f"{x} {y} {z} {a}" for (x, y, z), a in zip(s.xyz.tolist(), s.attributes.tolist())]
    for i in range(s.n):
        k = int(s.nbr_count[i])
        lines.append(" ".join([str(k)] + [str(int(v)) for v in s.nbr_ids[i, :k]]))
    lines.append(f"run {steps} {calls}")
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("build,steps,calls", [(S.small_chains, 50, 3), (S.square_network, 200, 2)])
def test_reference_adapter_over_engine_vs_oracle(build, steps, calls):
    """The reference's own LeMonADE adapter (src/pscbfm/GPUScBFM_AB_Type.h, compiled unchanged over
    include/bfm_updater.hpp into oracle/_ref/ref_adapter) drives the engine through its
    initialize/execute/cleanup: after `calls` execute() calls of `steps` MCS the positions equal the
    oracle's after steps x calls MCS of the engine's default counter stream (seed 0), and the
    molecules' age is steps x calls."""
    import os
    import subprocess
    import numpy as np
    from oracle import oracle as O
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_adapter")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/ref_adapter is built only where the reference sources are present")
    s = build()
    run = subprocess.run([exe], input=_adapter_input(s, steps, calls), capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    lines = run.stdout.strip().split("\n")
    got = np.array([[int(v) for v in ln.split()] for ln in lines[:s.n]])
    assert lines[s.n] == f"age {steps * calls}"
    want, _ = O.run(s, steps * calls, seed=0)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("repr_", [P.REPR_AUTO, P.REPR_GATHER])
def test_stats_tickets_across_paths(repr_):
    """Tickets taken after graph-path runs copy a counter snapshot on a publishing stream of their
    own (bond codes: the one the next replay's first check takes; gather representation: the one a
    node at the end of the replay takes); after other paths they read the counters directly. Mixed,
    back to back and repeated, every ticket equals a synchronous read after the same MCS."""
    s = S.serpentine_chains(64, 32, 0.3, seed=5)
    a = fresh()
    a.load_system(s, mode=P.MODE_GRAPH, representation=repr_)
    b = fresh()
    b.load_system(s, mode=P.MODE_GRAPH, representation=repr_)
    plan = [(P.MODE_GRAPH, 3), (P.MODE_LAUNCH, 2), (P.MODE_GRAPH, 5), (P.MODE_GRAPH, 0), (P.MODE_GRAPH, 1),
            (P.MODE_LAUNCH, 1), (P.MODE_GRAPH, 2)]
    tickets, done = [], []
    total = 0
    for mode, n in plan:
        a.set_mode(mode)
        if n:
            a.run_async(n)
        total += n
        tickets.append(a.stats_async())
        done.append(total)
    got = [a.stats_wait(t) for t in tickets]
    k = 0
    for want_mcs, g in zip(done, got):
        b.runSimulationOnGPU(want_mcs - k)
        k = want_mcs
        assert g == b.stats() and g["mcs"] == want_mcs
    a.close()
    b.close()


def test_stats_tickets_in_flight_and_around_other_work():
    """Tickets taken after graph replays of bond-code systems wait for the next replay's snapshot
    (its first check takes it) or, when other work comes first or the ticket is waited for, read
    the counters directly. Steps queued two ahead of the wait, as a serving loop does, two tickets
    with no work between them, a timed kernel pass, a LAUNCH-path run and a Batch run between
    replays: every ticket equals a synchronous read after the same MCS."""
    import numpy as np
    s = S.serpentine_chains(64, 32, 0.3, seed=5)
    a = fresh()
    a.load_system(s, mode=P.MODE_GRAPH)
    b = fresh()
    b.load_system(s, mode=P.MODE_GRAPH)
    got, done, total = [], [], 0

    def ticket():
        done.append(total)
        return a.stats_async()

    pending = []
    for k in range(12):                    # one MCS per step, the counters read two steps later
        a.run_async(1)
        total += 1
        pending.append(ticket())
        if len(pending) > 2:
            got.append(a.stats_wait(pending.pop(0)))
    got += [a.stats_wait(t) for t in pending]
    t1, t2 = ticket(), ticket()            # no work between them
    a.run_async(3)
    total += 3
    t3 = ticket()
    a.time_kernels(2)                      # kernels timed one at a time change the counters too
    total += 2
    t4 = ticket()
    a.set_mode(P.MODE_LAUNCH)
    a.run_async(2)
    total += 2
    a.set_mode(P.MODE_GRAPH)
    a.run_async(1)
    total += 1
    t5 = ticket()
    other = fresh()
    other.load_system(S.small_chains(), mode=P.MODE_GRAPH)
    batch = P.Batch([a, other])
    batch.run(2)
    total += 2
    t6 = ticket()
    a.run_async(70)                        # more than one graph chunk
    total += 70
    t7 = ticket()
    got += [a.stats_wait(t) for t in (t1, t2, t3, t4, t5, t6, t7)]
    batch.close()
    other.close()
    k = 0
    for want_mcs, g in zip(done, got):
        if want_mcs > k:
            b.runSimulationOnGPU(want_mcs - k)
            k = want_mcs
        assert g == b.stats() and g["mcs"] == want_mcs, (want_mcs, g, b.stats())
    assert np.array_equal(a.get_coords(), b.get_coords())
    a.close()
    b.close()


def test_persistent_barrier_timeout_is_reported():
    """A persistent launch whose grid barrier cannot complete (injected on the host: the arrival
    count starts where no barrier's target is reached) ends at the barrier's time limit, the run
    reports the timeout, and the device stays usable for the next system."""
    import time
    import numpy as np
    from oracle import oracle as O
    s = S.small_chains()
    u = fresh()
    u.load_system(s, mode=P.MODE_PERSISTENT)
    u.inject_barrier_stall()
    t = time.perf_counter()
    with pytest.raises(P.BfmCudaError, match="timed out"):
        u.runSimulationOnGPU(3)
    assert time.perf_counter() - t < 60
    u.close()
    v = fresh()
    v.load_system(s, mode=P.MODE_PERSISTENT)
    v.runSimulationOnGPU(20)
    want, _ = O.run(s, 20)
    assert np.array_equal(v.get_coords(), want)
    v.close()


def test_auto_mode_picks_the_path_by_size():
    """AUTO: resident for a system whose largest colour group is at most 2048, a cluster of CTAs for
    systems its shared memory holds at 48 chunks of 32 per CTA, the persistent sweep for larger
    bond-code systems, the graph of launches for the 1M-monomer melt and for systems without bond
    codes."""
    import numpy as np
    cases = [(S.serpentine_chains(32, 32, 0.3, seed=3), P.MODE_RESIDENT), (S.small_chains(), P.MODE_CLUSTER),
             (S.crosslinked_network(), P.MODE_CLUSTER),
             (S.serpentine_chains(64, 64, 0.8, seed=13), P.MODE_CLUSTER),
             (S.serpentine_chains(128, 64, 0.23, seed=5), P.MODE_PERSISTENT),   # 59 chunks per CTA of 16
             (S.serpentine_chains(128, 64, 0.3, seed=3), P.MODE_PERSISTENT), (S.dense_melt(), P.MODE_GRAPH)]
    for s, want in cases:
        u = fresh()
        u.load_system(s)
        assert u.path() == want, s.name
        u.close()
    # a bond listed in one direction only: no bond codes, so no persistent sweep
    xyz = np.array([[2 * j, 0, 0] for j in range(16)])
    s = S.from_bonds((128, 128, 128), xyz, [(j, j + 1) for j in range(15)], seed=8)
    s.nbr_count = s.nbr_count.copy()
    s.nbr_count[5] = 1
    u = fresh()
    u.load_system(s)
    assert u.representation() == 0 and u.path() == P.MODE_GRAPH
    u.set_mode(P.MODE_PERSISTENT)
    assert u.path() == P.MODE_GRAPH      # a mode the system cannot use falls back to the graph
    u.close()


def test_stats_read_without_waiting_for_later_work():
    """bfm_stats_enqueue / bfm_stats_wait: each ticket gives the counters as they stood when it was
    queued, while later runs stay queued; the counters equal a synchronous read after the same MCS
    on an identical system; tickets older than the last 8 are refused."""
    s = S.small_chains()
    a = fresh()
    a.load_system(s, mode=P.MODE_GRAPH)
    b = fresh()
    b.load_system(s, mode=P.MODE_GRAPH)
    tickets = []
    for _ in range(3):
        a.run_async(4)
        tickets.append(a.stats_async())
    a.run_async(50)   # queued behind the third copy
    seen = []
    for t in tickets:
        seen.append(a.stats_wait(t))
    for k, got in enumerate(seen):
        b.runSimulationOnGPU(4)
        want = b.stats()
        assert got == want and got["mcs"] == 4 * (k + 1)
    a.synchronize()
    assert a.stats()["mcs"] == 62
    for _ in range(8):
        a.stats_async()
    with pytest.raises(ValueError):
        a.stats_wait(tickets[0])
    with pytest.raises(ValueError):
        a.stats_wait(0)
    a.close()
    b.close()
