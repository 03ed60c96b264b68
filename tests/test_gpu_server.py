"""The job server: each job's result (final positions and every observable sample) equals running
it alone; admission respects the memory budget; cancel, malformed jobs and a dying worker are
handled on the host without hanging."""
import numpy as np
import pytest

import pscbfm_b200 as P
from pscbfm_b200 import systems as S

pytestmark = pytest.mark.gpu


def alone(s, n_mcs, every):
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    samples = []
    done = 0
    while done < n_mcs:
        step = min(every - done % every, n_mcs - done)
        u.runSimulationOnGPU(step)
        done += step
        samples.append(u.observables_raw())
    xyz = u.get_coords().copy()
    n_mol = len(u.molecule_sizes())
    u.close()
    return xyz, np.stack(samples), n_mol


def test_results_equal_alone_in_the_mix():
    systems = S.ensemble(n_systems=10, base_seed=500)
    systems.append(S.rings_and_free())
    plan = [(s, 30 + 17 * i, 10 + (i % 3) * 7) for i, s in enumerate(systems)]
    srv = P.Server(0, budget_bytes=8 << 30)
    jobs = [srv.submit(s, n, k) for s, n, k in plan]
    for j in jobs:
        srv.wait(j, 300)
        assert srv.status(j) == P.Server.DONE
    for j, (s, n, k) in zip(jobs, plan):
        want_xyz, want_samples, n_mol = alone(s, n, k)
        xyz, samples, lat = srv.result(j)
        assert samples.shape[1] == 5 * n_mol + 513
        assert np.array_equal(xyz, want_xyz), s.name
        assert np.array_equal(samples, want_samples), s.name
        assert lat > 0
    times = [srv.job_times(j) for j in jobs]
    assert any(s1 < f0 and s0 < f1 for (_, s0, f0) in times for (_, s1, f1) in times if f0 != f1)
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["p99_s"] >= st["p50_s"] > 0
    assert st["resident_bytes"] == 0
    srv.close()


def test_late_arrival_joins_running_batch():
    import time
    srv = P.Server(0, budget_bytes=8 << 30)
    a = srv.submit(S.small_chains(), 20000, 1000)
    while srv.status(a) == P.Server.PENDING:
        time.sleep(0.001)
    b = srv.submit(S.serpentine_chains(32, 16, 0.3, seed=9), 200, 100)
    srv.wait(b, 120)
    assert srv.status(a) == P.Server.RUNNING          # b was admitted and left while a ran
    _, sa, _ = srv.job_times(a)
    _, sb, fb = srv.job_times(b)
    assert sa < sb < fb
    srv.wait(a, 300)
    fa = srv.job_times(a)[2]
    assert fb < fa
    want, _, _ = alone(S.serpentine_chains(32, 16, 0.3, seed=9), 200, 100)
    assert np.array_equal(srv.result(b)[0], want)
    srv.close()


def test_budget_refusal_and_queueing():
    big = S.dense_melt()
    est = P.Server.estimate_bytes(big)
    assert est > big.n * 40
    srv = P.Server(0, budget_bytes=est - 1)
    with pytest.raises(P.BfmBudgetError):
        srv.submit(big, 1, 1)
    srv.close()
    # a budget that holds one job at a time: all still finish, in arrival order
    small = [S.serpentine_chains(32, 16, 0.3, seed=70 + i) for i in range(4)]
    one = max(P.Server.estimate_bytes(s) for s in small)
    srv = P.Server(0, budget_bytes=one + one // 2)
    jobs = [srv.submit(s, 40, 10) for s in small]
    times = []
    for j in jobs:
        srv.wait(j, 120)
        assert srv.status(j) == P.Server.DONE
        times.append(srv.job_times(j))
    for (a0, s0, f0), (a1, s1, f1) in zip(times, times[1:]):
        assert a0 <= a1 and s1 >= f0    # in arrival order, each admitted after the previous left
    for a, s, f in times:
        assert a <= s <= f
    want, _, _ = alone(small[-1], 40, 10)
    assert np.array_equal(srv.result(jobs[-1])[0], want)
    srv.close()


@pytest.mark.parametrize("build", [S.small_chains, S.crosslinked_network, S.rings_and_free, S.dense_melt,
                                   lambda: S.serpentine_chains(64, 64, 0.4, seed=13)])
def test_estimate_covers_the_arena(build):
    """Admission charges at least what the system's arena takes on the device."""
    s = build()
    u = P.UpdaterGPUScBFM_AB_Type(0).load_system(s)
    assert P.Server.estimate_bytes(s) >= u.device_bytes()
    u.close()


def test_cancel_pending_and_running():
    srv = P.Server(0, budget_bytes=8 << 30, max_jobs=1)
    a = srv.submit(S.small_chains(), 200000, 100000)   # long: occupies the only slot
    b = srv.submit(S.small_chains(), 10, 5)            # waits for the slot
    srv.cancel(b)
    assert srv.status(b) == P.Server.CANCELLED
    srv.cancel(a)
    srv.wait(a, 120)
    assert srv.status(a) == P.Server.CANCELLED
    with pytest.raises(RuntimeError):
        srv.result(a)
    assert srv.stats()["resident_bytes"] == 0
    srv.close()


def test_malformed_jobs_fail_at_submit():
    srv = P.Server(0, budget_bytes=1 << 30)
    setup = P.UpdaterGPUScBFM_AB_Type(0)
    setup.setNrOfAllMonomers(2)                      # no box, no bond set
    with pytest.raises(RuntimeError, match="setLatticeSize"):
        srv.submit_setup(setup, 10, 5, n=2)
    s = S.small_chains()
    setup2 = P.UpdaterGPUScBFM_AB_Type(0)
    setup2.load_system(s, initialize=False)
    setup2.copyBondSet(3, 1, 0, True)
    with pytest.raises(RuntimeError, match="108"):
        srv.submit_setup(setup2, 10, 5, n=s.n)
    with pytest.raises(ValueError):
        srv.submit(s, 0, 5)
    srv.close()


def test_worker_death_is_reported():
    srv = P.Server(0, budget_bytes=8 << 30, max_jobs=1)
    a = srv.submit(S.small_chains(), 500000, 100000)
    srv.inject_fault(1)
    srv.wait(a, 60)                                   # returns: the job failed with the worker
    assert srv.status(a) == P.Server.FAILED
    with pytest.raises(RuntimeError, match="worker has stopped"):
        srv.submit(S.small_chains(), 10, 5)
    srv.close()
