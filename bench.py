#!/usr/bin/env python
"""Benchmark of the BFM sweep engine: attempted monomer moves/s (MCS x N / t) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one Monte Carlo step (every colour group once) of the workload's system(s), inputs
resident in HBM. Workloads (synthetic, generated from their sizes; no dataset is involved):
  dense_melt  (default) periodic 256^3, 16,384 chains x 64 (N = 1,048,576, phi = 0.5), seed 7
  small       periodic 64^3, 256 chains x 32 (N = 8192, phi = 0.25), seed 42
  network     periodic 128^3, 512 six-functional nodes + 1536 strands of 7 (N = 11,264), seed 3
  ensemble    256 systems, box {32,64,128}, chains {16..256}, phi U[0.1,0.5], batched
Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events on the engine's
stream, with the L2 flushed (a 256 MiB write) before every step; max over ranks. One process per
GPU under torchrun; a single system does not shard, so N GPUs run N replicas (weak scaling).

--impl reference times the reference's algorithm on the host cores: the CPU restatement of the
reference sweep (oracle/), one replica per core, same metric and workload; beside it
(`reference_gpu`) the reference's own GPU updater, compiled from its sources into oracle/_ref, on
the same workload and GPU. The main arm carries the same reference-updater leg for the three
single-system workloads as a baseline beside its own numbers (never as the measured path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["dense_melt", "small", "network", "ensemble"], default="dense_melt")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-cores", type=int, default=0, help="host processes of the CPU legs (0: all cores)")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched-vs-plain side measurement")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    return a


# ------------------------------------------------------------------ workloads

def build_workload(name):
    from pscbfm_b200 import systems as S
    if name == "dense_melt":
        return [S.dense_melt()]
    if name == "small":
        return [S.small_chains()]
    if name == "network":
        return [S.crosslinked_network()]
    return S.ensemble()


def workload_config(name, systems):
    if name == "dense_melt":
        return {"workload": "dense_melt_256^3_16384x64_phi0.5", "box": 256, "chains": 16384, "chain_length": 64,
                "monomers": systems[0].n, "seed": 7}
    if name == "small":
        return {"workload": "chains_64^3_256x32_phi0.25", "box": 64, "chains": 256, "chain_length": 32,
                "monomers": systems[0].n, "seed": 42}
    if name == "network":
        return {"workload": "network_128^3_512x6func_strands7", "box": 128, "monomers": systems[0].n, "seed": 3}
    return {"workload": "ensemble_256_systems", "systems": len(systems), "monomers": sum(s.n for s in systems),
            "seeds": "1000+i", "generator_seed": 20240611}


# ------------------------------------------------------------------ algorithmic bytes (roofline)

E2E_IN_FLIGHT = 2               # steps queued ahead of the one whose counters the e2e loop reads

# dependent L2 round trips of one sub-step on the grid path (the latency model of the roofline)
CHECK_ROUND_TRIPS = 3          # step entry -> lattice address and bond code -> occupancy words
PERFORM_ROUND_TRIPS = 2        # list lengths, entries and targets -> code, neighbour refs, temporary words


def check_bytes_per_move(systems, p_chk, code_mode):
    """Algorithmic bytes of one attempted move in the check kernel.

    Gather representation (code_mode 0): own xyz 12 B, per neighbour 4 B id + 12 B xyz, neighbour
    count 1 B, flag write 1 B, 9 occupancy bits, one temporary bit per tentative move.
    Bond codes (code_mode 1: 4 B words, 2: 8 B words): lattice address 4 B + code word, 9
    occupancy bits; per tentative move a 4 B mover-list entry, its 4 B target address and one
    temporary bit set."""
    n = sum(s.n for s in systems)
    kbar = sum(int(s.nbr_count.sum()) for s in systems) / n
    if code_mode == 0:
        return 12 + 16 * kbar + 1 + 1 + 9 / 8 + p_chk / 8, kbar
    w = 4 if code_mode == 1 else 8
    return 4 + w + 9 / 8 + p_chk * (8 + 1 / 8), kbar


def perform_bytes_per_move(kbar, p_chk, p_acc, code_mode):
    """Algorithmic bytes of one attempted move in the perform kernel (bond codes), which walks only
    the mover lists: per tentative move its list entry 4 B, its target address 4 B, its code word,
    kbar neighbour references (4 B) and 9 temporary-lattice bits; per tentative move of the
    previous sub-step (the scrub, same rate) its target address 4 B and one temporary bit
    cleared; per accepted move 2 lattice bits read and written, the new lattice address 4 B, the
    own code word written and kbar neighbour code words read and written (the coordinates are image
    offsets, written only when a move wraps a periodic axis, about one move in a lattice side
    along that axis, and not counted). Gather representation (code_mode 0): flag 1 B, per tentative move xyz 12 B and 9
    temporary bits, per accepted move 2 lattice bits read and written, one coordinate 8 B, flag
    1 B."""
    if code_mode == 0:
        return 1 + p_chk * (12 + 9 / 8) + p_acc * (0.5 + 8 + 1)
    w = 4 if code_mode == 1 else 8
    return p_chk * (8 + w + 4 * kbar + 9 / 8) + p_chk * (4 + 1 / 8) + p_acc * (0.5 + 4 + w + 2 * w * kbar)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel_key, tag="dram_bytes_per_launch:"):
    """A figure recorded from an ncu capture in profiles/<kernel_key>.md (the line starting with
    tag: DRAM bytes per launch by default), if present."""
    p = os.path.join(ROOT, "profiles", kernel_key + ".md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.strip().startswith(tag):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------ clocks

class NvmlClockSampler:
    """SM clock and throttle reasons read through NVML every millisecond on a background thread
    (read only; nothing is set)."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, gpu_index):
        import threading
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(int(gpu_index))
        self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        self.samples, self.reasons = [], set()
        self.stop_flag = threading.Event()
        self.t = threading.Thread(target=self._loop, daemon=True)
        self.t.start()

    def _loop(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, const in self.REASONS.items():
                    if bits & getattr(nv, const):
                        self.reasons.add(name)
            except Exception:
                pass
            self.stop_flag.wait(0.001)

    def stop(self):
        self.stop_flag.set()
        self.t.join(timeout=2)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "sm_mhz_min": min(self.samples) if self.samples else None, "source": "nvml, every 1 ms"}


def clock_sampler(gpu_index):
    try:
        return NvmlClockSampler(gpu_index)
    except Exception:
        return ClockSampler(gpu_index)


class ClockSampler:
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + ",".join(self.FIELDS),
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [ln.split(", ") for ln in open(self.f.name).read().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU legs (oracle, spawned)

def _cpu_worker(args):
    kind, workload, steps, warmup = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    systems = build_workload(workload)
    s = systems[0] if workload != "ensemble" else max(systems, key=lambda q: q.n)
    attempted = 0
    t_total = 0.0
    seed = s.seed
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        if kind == "sequential":
            _, st = O.seq_run(s, 1, seed=seed + k)
            att = st[0]
        else:
            nc = int(O.color(s).max()) + 1
            _, st = O.run(s, 1, substep0=k * nc)
            att = st[0]
        dt = time.perf_counter() - t0
        if k >= warmup:
            attempted += att
            t_total += dt
    return attempted, t_total, s.n


def cpu_replicas(kind, workload, steps, warmup, cores=0):
    import multiprocessing as mp
    cores = cores or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(kind, workload, steps, warmup)] * cores)
    rate = sum(a / t for a, t, _ in res)
    return rate, cores, res[0][2]


def cpu_per_core(rate, cores):
    return rate / max(cores, 1)


# ------------------------------------------------------------------ main arm

def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, world, local


def _all_reduce(x, world, op):
    """One float across the ranks (CUDA tensor under NCCL, host tensor under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x, world):
    import torch.distributed as dist
    return _all_reduce(x, world, dist.ReduceOp.MAX)


def reduce_sum(x, world):
    import torch.distributed as dist
    return _all_reduce(x, world, dist.ReduceOp.SUM)


def aggregate_rate(units_per_rank, seconds_per_rank, world):
    """Whole-job throughput of weak-scaled replicas: units of all ranks / the slowest rank's time."""
    return reduce_sum(units_per_rank, world) / reduce_max(seconds_per_rank, world)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        parts = [p for p in vis.split(",") if p]
        if local < len(parts):
            return parts[local]
    return str(local)


def run_ours(args):
    import torch
    import pscbfm_b200 as P
    rank, world, local = dist_setup(args)
    systems = build_workload(args.workload)
    config = workload_config(args.workload, systems)
    n_total = sum(s.n for s in systems)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    members = [P.UpdaterGPUScBFM_AB_Type(local).load_system(s) for s in systems]
    colours = [m.n_colors()[0] for m in members]
    config = dict(config, colours=colours[0] if len(colours) == 1 else f"{min(colours)}-{max(colours)} per system")
    batch = P.Batch(members, gpu=local) if len(members) > 1 else None
    u0 = members[0]

    def step_timed(n):
        return u0.run_timed(n) if batch is None else batch.run_timed(n)

    def launch_count():
        return u0.launch_count() if batch is None else batch.launch_count()

    for _ in range(args.warmup):
        step_timed(1)
    launches0 = launch_count()
    stats0 = [m.stats() for m in members]
    barrier(world)
    torch.cuda.synchronize()
    sampler = clock_sampler(gpu_index(local))
    ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ms += step_timed(1)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier(world)
    launches = launch_count() - launches0
    stats1 = [m.stats() for m in members]
    attempted = sum(b["attempted"] - a["attempted"] for a, b in zip(stats0, stats1))
    tentative = sum(b["tentative"] - a["tentative"] for a, b in zip(stats0, stats1))
    accepted = sum(b["accepted"] - a["accepted"] for a, b in zip(stats0, stats1))
    t_max = reduce_max(ms / 1e3, world)
    moves = args.steps * n_total
    value = aggregate_rate(moves, ms / 1e3, world)
    p_chk, p_acc = tentative / max(attempted, 1), accepted / max(attempted, 1)

    # warm-L2 back-to-back number (no flush), for reference
    warm_ms = step_timed(args.steps)
    value_warm = world * moves / reduce_max(warm_ms / 1e3, world)

    # roofline of the dominant kernel
    hbm_peak, peak_kind = measured_peaks()
    roofline = None
    if batch is None:
        kt = u0.time_kernels(max(4, min(args.steps, 40)))
        code_mode = u0.representation()
        nC = u0.n_colors()[0]
        att_per_launch = systems[0].n / nC
        b_check, kbar = check_bytes_per_move(systems, p_chk, code_mode)
        b_perf = perform_bytes_per_move(kbar, p_chk, p_acc, code_mode)
        avg_check = kt["check_ms"] / kt["check_launches"]
        avg_perform = kt["perform_ms"] / kt["perform_launches"]
        achieved = b_check * att_per_launch / (avg_check / 1e3) / 1e9
        achieved_perf = b_perf * att_per_launch / (avg_perform / 1e3) / 1e9
        kname = "k_check" if code_mode == 0 else "k_check_bc"
        key = kname + "_" + {"dense_melt": "dense_melt256", "small": "chains64",
                             "network": "network128"}[args.workload]
        traffic = profiled_traffic(key)
        roofline = {"kernel": "bfm::" + kname, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                    "unit": "GB/s", "frac": round(achieved / hbm_peak, 4), "peak_kind": peak_kind,
                    "traffic": traffic, "algorithmic_bytes_per_launch": round(b_check * att_per_launch),
                    "bytes_per_attempted_move": round(b_check, 3), "kbar": round(kbar, 5),
                    "representation": ["gather", "bond codes 32-bit", "bond codes 64-bit"][code_mode],
                    "avg_launch_us": round(avg_check * 1e3, 2),
                    "perform": {"kernel": "bfm::k_perform" + ("" if code_mode == 0 else "_bc"),
                                "avg_launch_us": round(avg_perform * 1e3, 2),
                                "bytes_per_attempted_move": round(b_perf, 3),
                                "achieved": round(achieved_perf, 1), "frac": round(achieved_perf / hbm_peak, 4)},
                    "timing": "CUDA events around each launch on the engine stream, one sub-step at a time",
                    "note": ("the state (about 40 B per monomer) stays in the 126 MB L2 between launches, so "
                             "the HBM fraction is low by construction; the kernels are bound by instruction "
                             "issue and dependent-load latency")}
        # measured in this run on this GPU: the L2's read bandwidth, its hit latency and the period of
        # back-to-back kernels of the grid-phase shape in a graph (bfm_probe_device)
        probe = P.probe_device(local)
        roofline["l2"] = {"achieved": round(achieved, 1), "peak": round(probe["l2_read_gbs"], 1), "unit": "GB/s",
                          "frac": round(achieved / probe["l2_read_gbs"], 4),
                          "peak_source": "bfm_probe_device: 32 MB read 20 times by every SM, this run"}
        # latency bound of one MCS: per sub-step the check's dependent L2 round trips (step entry ->
        # lattice address and code -> occupancy words) and the perform's (list lengths, entries and
        # targets -> code words, neighbour references and temporary-lattice words), each one L2 hit
        # latency, plus two kernel periods
        rt = CHECK_ROUND_TRIPS + PERFORM_ROUND_TRIPS
        bound_us = nC * (rt * probe["l2_latency_ns"] / 1e3 + 2 * probe["kernel_period_us"])
        warm_us = warm_ms * 1e3 / args.steps
        roofline["latency"] = {"bound_us_per_mcs": round(bound_us, 2), "measured_us_per_mcs": round(warm_us, 2),
                               "frac": round(bound_us / warm_us, 4), "l2_latency_ns": round(probe["l2_latency_ns"], 1),
                               "kernel_period_us": round(probe["kernel_period_us"], 3),
                               "round_trips_per_sub_step": rt, "sub_steps_per_mcs": nC,
                               "model": "sub-steps x (dependent L2 round trips x L2 hit latency + 2 kernel periods), "
                                        "against the warm-L2 device time per MCS"}

    # e2e through the C-ABI with host buffers: per step one run of 1 MCS and a read of that step's
    # move counters into host memory; the host queues steps t + 1 and t + 2 before it waits for
    # step t's counters, so two steps are in flight while it reads; the positions, in the caller's
    # order, copied back into a pinned host array at the end
    host_xyz = torch.empty((systems[0].n, 3), dtype=torch.int32, pin_memory=True).numpy()

    def e2e_steps(k):
        pending = []
        for _ in range(k):
            if batch is None:
                u0.run_async(1)
            else:
                batch.run_async(1)
            pending.append(u0.stats_async())
            if len(pending) > E2E_IN_FLIGHT:
                u0.stats_wait(pending.pop(0))
        for ticket in pending:
            u0.stats_wait(ticket)
        u0.get_coords(host_xyz)

    e2e_steps(args.warmup)   # untimed: the same calls, so first-use set-up stays out of the timing
    xfer0 = [m.transfer_bytes() for m in members]
    torch.cuda.synchronize()
    t = time.perf_counter()
    e2e_steps(args.steps)
    e2e_s = time.perf_counter() - t
    xfer1 = [m.transfer_bytes() for m in members]
    h2d = sum(b[0] - a[0] for a, b in zip(xfer0, xfer1))
    d2h = sum(b[1] - a[1] for a, b in zip(xfer0, xfer1))
    e2e_value = world * moves / reduce_max(e2e_s, world)
    e2e = {"value": e2e_value, "unit": "attempted moves/s",
           "h2d_bytes_per_step": round(h2d / args.steps, 1), "d2h_bytes_per_step": round(d2h / args.steps, 1),
           "h2d_bytes": h2d, "d2h_bytes": d2h,
           "calls": "bfm_run_async(1) + bfm_stats_enqueue per step (the three move counters written into "
                    "mapped host memory), bfm_stats_wait on the ticket of the step before the previous one "
                    "(two steps in flight), "
                    "bfm_get_coords_bulk once into pinned memory; byte counts from bfm_transfer_bytes. A "
                    "step's only input is its MCS count (a launch argument): the sub-step entries of the "
                    "counter draw stream are made on the device, and the first entry of the device's "
                    "chain went up during the untimed warm-up steps of the same calls"}

    for m in members:
        m.validate()   # excluded volume, bonds and the device lattice after the timed run
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras and args.workload != "ensemble":
        if batch is not None:
            batch.close()
        for m in members:
            m.close()
        members, batch = [], None
        extras["reference_gpu"] = reference_gpu(gpu=local)
        r = extras["reference_gpu"]["workloads"].get(args.workload, {})
        if "reference_device" in r:
            # the engine's numbers of this line against the reference updater's on this GPU
            extras["vs_reference_gpu"] = {"value": value / r["reference_device"],
                                          "value_warm_l2": value_warm / r["reference_device"],
                                          "e2e": e2e_value / r["reference_host_clock"],
                                          "note": "value and value_warm_l2 over the reference's device time (warm "
                                                  "L2, its own call shape); e2e over its host-clock rate"}
        extras["batched"] = batched_vs_plain()
        extras["served"] = served(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, _ = cpu_replicas("sequential", args.workload, steps=3 if n_total > 100000 else 40, warmup=1,
                                      cores=args.cpu_cores)
        cpu = {"value": rate, "unit": "attempted moves/s", "cores": cores, "per_core": cpu_per_core(rate, cores),
               "kind": "port",
               "sample": ("random-sequential single-monomer BFM (LeMonADE serial-updater scheme), one replica of "
                          "the workload system per core, " + ("3" if n_total > 100000 else "40") + " MCS each")}
    launches_total = reduce_sum(float(launches), world)
    if rank == 0:
        line = {"metric": "attempted monomer moves/s", "value": value, "unit": "attempted moves/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": dict(config, l2="flushed (256 MiB write) before every timed step",
                               path="auto" if batch is None else "batch", parallelism=f"replicas x{world}"),
                "value_warm_l2": value_warm, "p_chk": p_chk, "p_acc": p_acc,
                "moves_timed": {"attempted": attempted, "tentative": tentative, "accepted": accepted,
                                "sub_steps": args.steps * sum(colours)},
                "l2_cache_bytes": torch.cuda.get_device_properties(local).L2_cache_size,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches_total),
                "clocks": clocks}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


ENSEMBLE_MCS = 10000
REFERENCE_LONG = os.path.join(ROOT, "tests", "golden", "reference_long.json")


def positions_sha256(xyz):
    import hashlib
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(np.asarray(xyz, dtype="<i4").reshape(-1, 3)).tobytes()).hexdigest()


def plain_rates(systems, sample_mcs, gpu=0, every=None, mcs_cap=None):
    """Each system alone, one after another, on the plain paths: BFM_MODE_LAUNCH (two launches per
    sub-step, the reference's structure) and BFM_MODE_AUTO (the engine's own choice for one system:
    resident, cluster, persistent or graph). Per system 3 untimed MCS, then min(sample_mcs, its MCS)
    timed (CUDA events; with `every`, observables read back every `every` MCS as the server does, on
    the host clock). Returns per mode the attempted moves and seconds of the timed samples."""
    import pscbfm_b200 as P
    out = {}
    for name, mode in (("launch", P.MODE_LAUNCH), ("auto", P.MODE_AUTO)):
        moves, secs = 0, 0.0
        for i, sy in enumerate(systems):
            k = sample_mcs if mcs_cap is None else min(sample_mcs, mcs_cap[i])
            u = P.UpdaterGPUScBFM_AB_Type(gpu).load_system(sy, mode=mode)
            u.runSimulationOnGPU(3)
            if every is None:
                secs += u.run_timed(k) / 1e3
            else:
                u.synchronize()
                t = time.perf_counter()
                done = 0
                while done < k:
                    step = min(every - done % every, k - done)
                    u.runSimulationOnGPU(step)
                    done += step
                    if done % every == 0:
                        u.observables_raw()
                secs += time.perf_counter() - t
            moves += sy.n * k
            u.close()
        out[name] = (moves, secs)
    return out


def batched_vs_plain(mcs=ENSEMBLE_MCS, sample_mcs=200):
    """The 256-system ensemble (own seeds 1000 + i) in one Batch for its full 10^4 MCS: the run's first
    MCS are the autotuner's trials, then a timed sample of sample_mcs MCS, then the rest of the run
    timed; every member's final positions are compared with the reference updater's run of that
    system alone (tests/golden/reference_long.json). Beside it the same systems one at a time on the
    two plain paths over a timed sample of sample_mcs MCS each (plain_rates). Rates are measured, not
    extrapolated: attempted moves / device seconds of each timed region."""
    import json
    import pscbfm_b200 as P
    from pscbfm_b200 import systems as S
    systems = S.ensemble(n_systems=256)
    n = sum(s.n for s in systems)
    members = [P.UpdaterGPUScBFM_AB_Type(0).load_system(s) for s in systems]
    b = P.Batch(members)
    b.run(3)
    tuned = b.autotune(2)          # the trials are MCS of the run
    done = 3 + tuned["mcs_spent"]
    sample_ms = b.run_timed(sample_mcs)
    launches0 = b.launch_count()
    rest = mcs - done - sample_mcs
    rest_ms = b.run_timed(rest)
    launches_per_mcs = (b.launch_count() - launches0) / rest
    b.synchronize()
    parity = {"checked": False}
    if os.path.exists(REFERENCE_LONG):
        gold = json.load(open(REFERENCE_LONG))["cases"]
        same = sum(positions_sha256(m.get_coords()) == gold[f"ensemble256_{i:03d}_{mcs}mcs"]["sha256"]
                   for i, m in enumerate(members))
        parity = {"checked": True, "members_equal_reference": int(same), "members": len(members),
                  "mcs": mcs, "against": "reference updater run on each system alone (reference_long.json)"}
    for m in members:
        m.validate()
    b.close()
    for m in members:
        m.close()
    plain = plain_rates(systems, sample_mcs)
    batched_sample = n * sample_mcs / (sample_ms / 1e3)
    batched_long = n * rest / (rest_ms / 1e3)
    rate = {k: v[0] / v[1] for k, v in plain.items()}
    return {"workload": "ensemble_256_systems", "systems": len(systems), "monomers": n, "mcs": mcs,
            "batched": batched_long, "batched_sample": batched_sample,
            "plain_launch": rate["launch"], "plain_auto": rate["auto"],
            "ratio_vs_plain_launch": batched_sample / rate["launch"],
            "ratio_vs_plain_auto": batched_sample / rate["auto"],
            "batched_launches_per_mcs": launches_per_mcs, "parity": parity,
            "autotuned": {"shape": tuned["shape"], "resident": tuned["resident"], "cluster": tuned["cluster"],
                          "block": tuned["block"], "perform": list(tuned["perform"]),
                          "trials": [[t["shape"], t["resident"], t["cluster"], t["block"], list(t["perform"]),
                                      round(t["ms_per_mcs"], 4)] for t in tuned["trials"]],
                          "trial_fields": ["shape", "resident", "cluster", "block",
                                           "perform (warps per CTA, per tile; 0 = default 4)", "ms_per_mcs"]},
            "timing": (f"batched: CUDA events over MCS {done}-{done + sample_mcs} (batched_sample, compared with "
                       f"the plain samples) and {done + sample_mcs}-{mcs} (batched); plain: each system alone, "
                       f"CUDA events over its MCS 3-{3 + sample_mcs}"),
            "unit": "attempted moves/s"}


SERVED_RATES = (10, 30, 100, 300, 1000)


def served_jobs(n_jobs, seed=777):
    """The served job set: systems drawn like the batched ensemble (own seeds), MCS log-uniform on
    [1e3, 1e5], observables every 100 MCS."""
    import numpy as np
    from pscbfm_b200 import systems as S
    systems = S.ensemble(n_systems=n_jobs, base_seed=50000, gen_seed=seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    mcs = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n_jobs)).astype(np.int64)
    return systems, [int(m) for m in mcs]


def served(gpu=0, n_jobs=200, rates=SERVED_RATES, budget=150 << 30, every=100, sample_mcs=300):
    """Poisson arrivals at each rate lambda of n_jobs jobs into the job server (HBM budget 150 GB,
    observables every 100 MCS); latency = submit to completion on the host clock. Beside it the
    same jobs one at a time on the two plain paths (plain_rates: min(MCS, sample_mcs) MCS of each
    job timed with the same observable sampling); the ratios compare measured rates."""
    import numpy as np
    import pscbfm_b200 as P
    systems, mcs = served_jobs(n_jobs)
    work = sum(s.n * m for s, m in zip(systems, mcs))
    longest = int(np.argmax([s.n * m for s, m in zip(systems, mcs)]))
    setups = [P.UpdaterGPUScBFM_AB_Type(gpu).load_system(s, initialize=False) for s in systems]
    plain = plain_rates(systems, sample_mcs, gpu=gpu, every=every, mcs_cap=mcs)
    rate = {k: v[0] / v[1] for k, v in plain.items()}
    rows = []
    for lam in rates:
        rng = np.random.Generator(np.random.PCG64(int(lam)))
        arrivals = np.cumsum(rng.exponential(1.0 / lam, n_jobs))
        srv = P.Server(gpu, budget_bytes=budget)
        t0 = time.perf_counter()
        jobs = []
        for a, u, s, m in zip(arrivals, setups, systems, mcs):
            dt = t0 + a - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            jobs.append(srv.submit_setup(u, m, every, n=s.n))
        for j in jobs:
            srv.wait(j, 900)
        makespan = time.perf_counter() - t0
        st = srv.stats()
        lat_longest = srv.job_times(jobs[longest])
        srv.close()
        if st["completed"] != n_jobs:
            raise RuntimeError(f"served: {st['completed']} of {n_jobs} jobs completed")
        moves_per_s = work / makespan
        rows.append({"lambda_jobs_per_s": lam, "p50_s": round(st["p50_s"], 4), "p99_s": round(st["p99_s"], 4),
                     "mean_s": round(st["mean_s"], 4), "makespan_s": round(makespan, 3), "moves_per_s": moves_per_s,
                     "ratio_vs_plain_launch": moves_per_s / rate["launch"],
                     "ratio_vs_plain_auto": moves_per_s / rate["auto"],
                     "longest_job_share_of_makespan": round((lat_longest[2] - lat_longest[0]) / makespan, 4)})
    for u in setups:
        u.close()
    return {"jobs_per_rate": n_jobs, "monomers_x_mcs": work, "every": every, "budget_bytes": budget,
            "plain_launch": rate["launch"], "plain_auto": rate["auto"], "rates": rows,
            "longest_job": {"monomers": systems[longest].n, "mcs": mcs[longest], "box": list(systems[longest].box)},
            "unit": "attempted moves/s", "clock": "host wall clock, submit to completion",
            "plain": (f"each job alone on BFM_MODE_LAUNCH and on BFM_MODE_AUTO with observables every {every} MCS; "
                      f"min(MCS, {sample_mcs}) MCS of each timed; rates = attempted moves / seconds of the samples")}


REFERENCE_GPU_RUNS = {"dense_melt": (10, 200), "small": (100, 1000), "network": (100, 1000)}


def reference_gpu(workloads=("dense_melt", "small", "network"), gpu=0, with_engine=True):
    """Baseline leg: the reference's own GPU updater (src/pscbfm, compiled for sm_100a from its
    sources into oracle/_ref by oracle/Makefile), timed on this GPU like its own tGpuLoop figure
    (CUDA events on the legacy default stream it runs on, around runSimulationOnGPU(n), after an
    untimed warm-up call), with the host clock of the same call beside it (the reference's MCS*N/t).
    Beside each, the engine through the same call shape: one runSimulationOnGPU(n) plus the read-back
    of the positions, host clock (with_engine; the reference arm runs the reference alone). Never the
    engine's measured path: a baseline, like cpu_baseline."""
    import numpy as np
    from oracle import oracle as O
    out = {}
    for w in workloads:
        s = build_workload(w)[0]
        warm, timed = REFERENCE_GPU_RUNS[w]
        conn = int(s.nbr_count.max())
        if not O.ref_available(s.walls, conn):
            out[w] = {"unavailable": "oracle/_ref not built (needs the reference sources at build time)"}
            continue
        # the reference's warm-up call is warm + timed MCS, so that after it both sides have run the
        # same sub-steps (the engine's warm-up is `warm` plus one timed run of `timed` MCS)
        ms, wall, ref_xyz = O.ref_time(s, warm + timed, timed, reps=1, gpu=gpu)
        moves = s.n * timed
        row = {"monomers": s.n, "warmup_mcs": warm + timed, "timed_mcs": timed,
               "reference_device": moves / (ms / 1e3), "reference_ms_per_mcs": ms / timed,
               "reference_host_clock": moves / wall,
               "reference_build": "MAX_CONNECTIVITY 8" if conn > 4 else "MAX_CONNECTIVITY 4"}
        out[w] = row
        if not with_engine:
            continue
        import pscbfm_b200 as P
        import torch
        u = P.UpdaterGPUScBFM_AB_Type(gpu).load_system(s)
        u.runSimulationOnGPU(warm)
        host = torch.empty((s.n, 3), dtype=torch.int32, pin_memory=True).numpy()
        ours_dev_ms = u.run_timed(timed)   # also captures the graphs a call of timed MCS replays
        t0 = time.perf_counter()
        u.runSimulationOnGPU(timed)
        u.get_coords(host)
        t_ours = time.perf_counter() - t0
        ours_xyz = host.copy()
        u.close()
        row.update({"engine_same_call_host_clock": moves / t_ours, "engine_device": moves / (ours_dev_ms / 1e3),
                    "ratio_device": (moves / (ours_dev_ms / 1e3)) / row["reference_device"],
                    "ratio_host_clock": (moves / t_ours) / row["reference_host_clock"],
                    "same_positions": bool(np.array_equal(ref_xyz, ours_xyz))})
    return {"unit": "attempted moves/s", "workloads": out,
            "how": ("reference: bfmref_time (oracle/ref_harness.cu), CUDA events on stream 0 around "
                    "runSimulationOnGPU(timed_mcs) after runSimulationOnGPU(warmup_mcs), block size 128 and "
                    "cudaMemset clearing (its stock settings); both include its copy-back of the positions. "
                    "engine: after the same warm-up MCS (the last timed_mcs of them timed by CUDA events: "
                    "engine_device), one runSimulationOnGPU(timed_mcs) plus bfm_get_coords_bulk into pinned "
                    "memory on the host clock (engine_same_call_host_clock); warm L2 on both sides; "
                    "same_positions compares the two after the same MCS")}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    systems = build_workload(args.workload)
    config = workload_config(args.workload, systems)
    steps = min(args.steps, 5 if sum(s.n for s in systems) > 100000 else 50)
    rate, cores, n = cpu_replicas("parallel", args.workload, steps=steps, warmup=min(args.warmup, 1),
                                  cores=args.cpu_cores)
    sample = (f"CPU restatement of the reference's colour-by-colour sweep (oracle/bfm_oracle.cpp), one "
              f"replica per core, {steps} MCS each after 1 warm-up MCS")
    ref_gpu = None
    if args.workload in REFERENCE_GPU_RUNS:
        try:
            ref_gpu = reference_gpu(workloads=(args.workload,), with_engine=False)
        except Exception as e:   # no GPU or no reference build: the CPU arm stands alone
            ref_gpu = {"unavailable": str(e).splitlines()[0][:200]}
    line = {"impl": "reference", "metric": "attempted monomer moves/s", "value": rate, "unit": "attempted moves/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config,
            "cpu_baseline": {"value": rate, "unit": "attempted moves/s", "cores": cores,
                             "per_core": cpu_per_core(rate, cores), "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "attempted moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
