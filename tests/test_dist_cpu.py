"""Multi-process paths on the CPU (gloo, world size 2): the bench's reductions over ranks, the
reference arm under torchrun, and sets of systems sharded over ranks with their results gathered
to rank 0. One system does not shard (one system is one replica), so N GPUs run N independent
replicas or N disjoint subsets of systems, and the only cross-rank steps are reductions and the
gather after the runs."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                           timeout=datetime.timedelta(seconds=60))
    import bench
    mx = bench.reduce_max(1.5 + rank, world)
    sm = bench.reduce_sum(2.0 * (rank + 1), world)
    # rank r processed 100 (r + 1) units in 0.5 (r + 1) s: aggregate = 300 units / 1.0 s
    rate = bench.aggregate_rate(100.0 * (rank + 1), 0.5 * (rank + 1), world)
    bench.barrier(world)
    q.put((rank, mx, sm, rate))
    dist.destroy_process_group()


def test_reductions_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, rate in got:
        assert mx == 2.5 and sm == 6.0
        assert rate == pytest.approx(300.0)


def _shard_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                           timeout=datetime.timedelta(seconds=60))
    from oracle import oracle as O
    from pscbfm_b200 import sharding
    systems, mcs = _shard_case()
    seen = []

    def run_local(ss, ms):
        seen.extend(s.name for s in ss)
        return [O.run(s, m)[0] for s, m in zip(ss, ms)]

    res = sharding.run_sharded(systems, mcs, run_local, rank=rank, world=world)
    q.put((rank, seen, None if res is None else [r.tolist() for r in res]))
    dist.destroy_process_group()


def _shard_case():
    from pscbfm_b200 import systems as S
    systems = [S.serpentine_chains(32, 16, 0.2 + 0.05 * k, name=f"shard{k}", seed=70 + k) for k in range(5)]
    systems.append(S.walled(S.serpentine_chains((24, 32, 20), 8, 0.3, seed=79), walls=5, name="shard5"))
    return systems, [40, 10, 25, 5, 30, 20]


def test_shard_systems_is_balanced_and_deterministic():
    sys.path.insert(0, ROOT)
    from pscbfm_b200.sharding import shard_systems
    costs = [5, 1, 4, 3, 3, 2, 8]
    a = shard_systems(costs, 3)
    assert a == shard_systems(costs, 3)
    assert sorted(i for part in a for i in part) == list(range(len(costs)))
    loads = [sum(costs[i] for i in part) for part in a]
    assert max(loads) - min(loads) <= max(costs)
    # in decreasing cost 8, 5, 4, 3, 3, 2, 1, each to the least-loaded rank (ties: the lower rank)
    assert a == [[1, 6], [0, 4], [2, 3, 5]]          # 8 + 1 | 5 + 3 | 4 + 3 + 2
    assert shard_systems([1.0, 1.0], 4) == [[0], [1], [], []]


def test_run_sharded_on_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from pscbfm_b200 import sharding
    systems, mcs = _shard_case()
    calls = []

    def run_local(ss, ms):
        calls.append(len(ss))
        return [(s.name, m) for s, m in zip(ss, ms)]

    out = sharding.run_sharded(systems, mcs, run_local)
    assert calls == [len(systems)]
    assert out == [(s.name, m) for s, m in zip(systems, mcs)]
    with pytest.raises(ValueError):
        sharding.run_sharded(systems, mcs[:-1], run_local)
    with pytest.raises(RuntimeError):
        sharding.run_sharded(systems, mcs, lambda ss, ms: [])


def test_sharded_runs_over_two_gloo_ranks_gather_to_rank0():
    """Two ranks split six systems by monomers x MCS, each runs its own (the oracle stands in for
    a rank's GPU), and rank 0 receives every system's final positions in the original order,
    equal to running each system alone."""
    import multiprocessing as mp
    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    systems, mcs = _shard_case()
    (_, seen0, res0), (_, seen1, res1) = got
    assert res1 is None and len(res0) == len(systems)
    assert seen0 and seen1 and sorted(seen0 + seen1) == sorted(s.name for s in systems)
    for s, m, r in zip(systems, mcs, res0):
        want, _ = O.run(s, m)
        assert np.array_equal(np.asarray(r), want), s.name


def test_reference_arm_under_torchrun_prints_one_line():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--workload", "small", "--cpu-cores", "2"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1          # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 2
