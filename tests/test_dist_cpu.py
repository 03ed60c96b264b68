"""Multi-process paths on the CPU (gloo, world size 2): the bench's reductions over ranks and the
reference arm under torchrun. The sweep does not shard (one system is one replica), so N GPUs
run N independent replicas and the only cross-rank steps are these reductions."""
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
