"""Python mirror of the reference updater interface over the C-ABI.

``UpdaterGPUScBFM_AB_Type`` keeps the method names, argument meaning and call order of
src/pscbfm/UpdaterGPUScBFM_AB_Type.h:316-358; errors raise the Python counterpart of the
reference's exception (std::invalid_argument -> ValueError, std::runtime_error -> RuntimeError,
std::out_of_range -> IndexError, CUDA errors -> BfmCudaError). ``Batch`` advances many updaters
together (no reference counterpart).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MODE_AUTO, MODE_GRAPH, MODE_LAUNCH, MODE_PERSISTENT, MODE_RESIDENT, MODE_CLUSTER  # noqa: F401

REPR_AUTO, REPR_GATHER = 0, 1


def color_graph(system) -> np.ndarray:
    """Colours of the system's monomers as initialize() computes them (host only, no GPU)."""
    L = _lib.load()
    cnt = np.ascontiguousarray(system.nbr_count, dtype=np.uint32)
    ids = np.ascontiguousarray(system.nbr_ids, dtype=np.uint32).reshape(-1)
    out = np.zeros(system.n, dtype=np.uint8)
    nc = C.c_uint32()
    st = L.bfm_color_graph(system.n, cnt, ids, system.maxc, out, C.byref(nc))
    if st != _lib.BFM_OK:
        _lib.raise_for(st, L.bfm_last_error(None).decode())
    return out


def probe_device(gpu: int = 0) -> dict:
    """bfm_probe_device: L2 hit latency, L2 read bandwidth and the period of back-to-back kernels of
    the grid-phase shape in a captured graph, measured on the GPU."""
    out = np.zeros(4, dtype=np.float64)
    st = _lib.load().bfm_probe_device(gpu, out)
    if st != _lib.BFM_OK:
        _lib.raise_for(st, "bfm_probe_device failed")
    return {"l2_latency_ns": float(out[0]), "l2_read_gbs": float(out[1]), "kernel_period_us": float(out[2]),
            "sms": int(out[3])}


def counter_draw(seed: int, k: int) -> int:
    return int(_lib.load().bfm_counter_draw(seed, k))


def decode_observables(raw: np.ndarray, sizes: np.ndarray) -> dict:
    """Splits the int64 words of bfm_observables and derives the float observables on the host."""
    m = len(sizes)
    mom = raw[:4 * m].reshape(m, 4)
    s1, s2 = mom[:, :3], mom[:, 3]
    ree2 = raw[4 * m:5 * m]
    hist = raw[5 * m:5 * m + 512]
    msd_sum = int(raw[5 * m + 512])
    n = sizes.astype(np.float64)
    rg2 = s2 / n - (s1.astype(np.float64) ** 2).sum(axis=1) / n ** 2
    return {"sum_r": s1, "sum_r2": s2, "ree2": ree2, "bond_hist": hist, "msd_sum": msd_sum, "sizes": sizes,
            "rg2": rg2, "rg2_mean": float(rg2.mean()), "ree2_mean": float(ree2.mean()),
            "msd": msd_sum / float(sizes.sum())}


class UpdaterGPUScBFM_AB_Type:
    def __init__(self, gpu: int = 0):
        self._L = _lib.load()
        h = C.c_void_p()
        self._check(self._L.bfm_create(C.byref(h), gpu), None)
        self._h = h
        self._draw_cb = None

    # ---------------------------------------------------------------- plumbing
    def _check(self, status, h="self"):
        if status != _lib.BFM_OK:
            handle = self._h if h == "self" else None
            _lib.raise_for(status, self._L.bfm_last_error(handle).decode())

    def _call(self, name, *args):
        self._check(getattr(self._L, name)(self._h, *args))

    def close(self):
        if getattr(self, "_h", None):
            self._L.bfm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------------- reference API
    def setGpu(self, gpu: int):
        self._call("bfm_set_gpu", gpu)

    def setPeriodicity(self, px: bool, py: bool, pz: bool):
        self._call("bfm_set_periodicity", int(px), int(py), int(pz))

    def setNrOfAllMonomers(self, n: int):
        self._call("bfm_set_n_monomers", n)
        self.n_monomers = n

    def setAttribute(self, i: int, attribute: int):
        self._call("bfm_set_attribute", i, attribute)

    def setMonomerCoordinates(self, i: int, x: int, y: int, z: int):
        self._call("bfm_set_coords", i, x, y, z)

    def setConnectivity(self, a: int, b: int):
        self._call("bfm_add_bond", a, b)

    def setLatticeSize(self, bx: int, by: int, bz: int):
        self._call("bfm_set_box", bx, by, bz)

    def copyBondSet(self, dx: int, dy: int, dz: int, forbidden: bool):
        self._call("bfm_set_bond_forbidden", dx, dy, dz, int(forbidden))

    def populateLattice(self):
        self._call("bfm_populate_lattice")

    def initialize(self):
        self._call("bfm_initialize")

    def execute(self) -> bool:
        return True

    def runSimulationOnGPU(self, n_mcs: int):
        self._call("bfm_run", n_mcs)

    def getMonomerPositionInX(self, i: int) -> int:
        return self._coord(i, 0)

    def getMonomerPositionInY(self, i: int) -> int:
        return self._coord(i, 1)

    def getMonomerPositionInZ(self, i: int) -> int:
        return self._coord(i, 2)

    def cleanup(self):
        self._call("bfm_cleanup")

    def _coord(self, i, axis):
        out = C.c_int32()
        self._call("bfm_get_coord", i, axis, C.byref(out))
        return out.value

    # ---------------------------------------------------------------- engine extensions
    def set_seed(self, seed: int):
        self._call("bfm_set_seed", seed)
        self._seed = int(seed)

    def set_substep(self, substep: int):
        """Position of the counter draw stream (after initialize), e.g. from a checkpoint."""
        self._call("bfm_set_substep", substep)

    def substep(self) -> int:
        v = C.c_uint64()
        self._call("bfm_get_substep", C.byref(v))
        return v.value

    def save_checkpoint(self, path: str, system):
        """Writes the current positions of `system`'s monomers to a .bfm file whose header holds the
        draw-stream position; load_checkpoint resumes from it bit-exactly."""
        from .bfm_io import write_bfm
        t = self.substep()
        write_bfm(path, system, mcs=t // self.n_colors()[0], xyz=self.get_coords(), substep=t,
                  seed=getattr(self, "_seed", 0))

    @classmethod
    def load_checkpoint(cls, path: str, system=None, gpu: int = 0, mode: int | None = None):
        """A new initialised updater at the state save_checkpoint wrote. Returns (updater, system).

        The colouring, like the reference's, depends on the order of each monomer's neighbour list,
        and a .bfm file fixes that order only as its reader rebuilds it (explicit bonds first, then
        the chain links). Pass the system the run started from to keep its order (positions come
        from the file); without it the file's own order is used, which continues bit-exactly only
        for systems that were themselves read from a .bfm file."""
        import dataclasses
        from .bfm_io import read_bfm
        read, info = read_bfm(path)
        if system is None:
            system = read
        else:
            if system.n != read.n or tuple(system.box) != tuple(read.box):
                raise ValueError("checkpoint does not match the given system (monomer count or box)")
            system = dataclasses.replace(system, xyz=read.xyz.astype(np.int32), seed=info["seed"])
        u = cls(gpu).load_system(system, seed=info["seed"], mode=mode)
        u.set_substep(info["substep"])
        return u, system

    def set_draw_callback(self, fn):
        """fn() -> int: an external host generator consumed twice per sub-step (colour, seed)."""
        cb = _lib.DRAW_FN(lambda _ctx: int(fn()) & 0xFFFFFFFF)
        self._draw_cb = cb
        self._call("bfm_set_draw_callback", cb, None)

    def set_grid_block(self, block: int):
        """CTA size of the bond-code check on the grid paths (128, 256, 512; 0 = default 256)."""
        self._call("bfm_set_grid_block", block)

    def set_perform(self, warps: int, group: int):
        """Warps per CTA and per tile of the bond-code perform on the grid paths (1, 2, 4, 8, group <=
        warps; 0, 0 = default 4, 4); results do not change."""
        self._call("bfm_set_perform", warps, group)

    def set_mode(self, mode: int):
        self._call("bfm_set_mode", mode)

    def set_standard_bond_set(self):
        self._call("bfm_set_standard_bond_set")

    def set_coords(self, xyz: np.ndarray):
        a = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1)
        self._call("bfm_set_coords_bulk", a, a.size // 3)

    def get_coords(self, out: np.ndarray | None = None) -> np.ndarray:
        n = self.n_monomers
        if out is None:
            out = np.empty((n, 3), dtype=np.int32)
        self._call("bfm_get_coords_bulk", out.reshape(-1), n)
        return out

    def run_async(self, n_mcs: int):
        self._call("bfm_run_async", n_mcs)

    def synchronize(self):
        self._call("bfm_synchronize")

    def path(self) -> int:
        """The engine path the next run takes (MODE_*): the set mode with MODE_AUTO resolved."""
        v = C.c_int()
        self._call("bfm_get_path", C.byref(v))
        return v.value

    def inject_barrier_stall(self):
        """Tests: the next persistent launch's grid barrier cannot complete; the run reports the
        timeout of its bounded wait (BfmCudaError) and the device stays usable."""
        self._call("bfm_inject_barrier_stall")

    def n_colors(self):
        n = C.c_uint32()
        self._call("bfm_n_colors", C.byref(n), None, 0)
        sizes = np.zeros(n.value, dtype=np.uint32)
        self._call("bfm_n_colors", C.byref(n), sizes.ctypes.data_as(C.c_void_p), n.value)
        return n.value, sizes

    def stats(self):
        """Move counters (waits for the handle's queued work): attempted, tentative, accepted, MCS."""
        out = self.__dict__.get("_stats_buf")
        if out is None:
            out = self._stats_buf = (C.c_uint64 * 4)()
        self._call("bfm_get_stats", out)
        return {"attempted": out[0], "tentative": out[1], "accepted": out[2], "mcs": out[3]}

    def stats_async(self) -> int:
        """Queues a copy of the move counters after the work queued so far; returns a ticket for
        stats_wait (the last 8 tickets stay valid)."""
        t = self.__dict__.get("_ticket_buf")
        if t is None:
            t = self._ticket_buf = C.c_uint64()
        self._call("bfm_stats_enqueue", C.byref(t))
        return t.value

    def stats_wait(self, ticket: int) -> dict:
        """The counters as they stood when the ticket was queued; waits for that copy only."""
        out = self.__dict__.get("_wait_buf")
        if out is None:
            out = self._wait_buf = (C.c_uint64 * 4)()
        self._call("bfm_stats_wait", ticket, out)
        return {"attempted": out[0], "tentative": out[1], "accepted": out[2], "mcs": out[3]}

    def validate(self):
        self._call("bfm_validate")

    def device_bytes(self) -> int:
        v = C.c_uint64()
        self._call("bfm_device_bytes", C.byref(v))
        return v.value

    def molecule_sizes(self) -> np.ndarray:
        n = C.c_uint32()
        self._call("bfm_n_molecules", C.byref(n))
        out = np.zeros(n.value, dtype=np.uint32)
        self._call("bfm_molecule_sizes", out, n.value)
        return out

    def observables_raw(self) -> np.ndarray:
        """The exact int64 words of bfm_observables (layout in include/bfm.h)."""
        n = C.c_uint32()
        self._call("bfm_n_molecules", C.byref(n))
        out = np.zeros(5 * n.value + 513, dtype=np.int64)
        self._call("bfm_observables", out, out.size)
        return out

    def observables(self) -> dict:
        """Exact sums plus the derived per-molecule Rg^2, Ree^2 and the mean squared displacement."""
        return decode_observables(self.observables_raw(), self.molecule_sizes())

    def reset_msd_reference(self):
        self._call("bfm_reset_msd_reference")

    def run_timed(self, n_mcs: int) -> float:
        """Runs n_mcs MCS; returns their device time in ms (CUDA events on the engine's stream)."""
        ms = C.c_float()
        self._call("bfm_run_timed", n_mcs, C.byref(ms))
        return ms.value

    def time_kernels(self, n_mcs: int):
        out = np.zeros(4, dtype=np.float64)
        self._call("bfm_time_kernels", n_mcs, out)
        return {"check_ms": out[0], "perform_ms": out[1], "check_launches": int(out[2]),
                "perform_launches": int(out[3])}

    def transfer_bytes(self) -> tuple:
        """(host -> device, device -> host) bytes of the run and read-back calls so far."""
        v = (C.c_uint64 * 2)()
        self._call("bfm_transfer_bytes", v)
        return int(v[0]), int(v[1])

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._call("bfm_launch_count", C.byref(v))
        return v.value

    n_monomers = 0

    def set_representation(self, repr_: int):
        """REPR_AUTO (bond codes where possible) or REPR_GATHER; before initialize()."""
        self._call("bfm_set_representation", repr_)

    def representation(self) -> int:
        v = C.c_int()
        self._call("bfm_get_representation", C.byref(v))
        return v.value

    def load_system(self, system, seed: int | None = None, mode: int | None = None, initialize: bool = True,
                    representation: int | None = None):
        """Feeds a systems.BfmSystem through the setter API in the adapter's order
        (src/pscbfm/GPUScBFM_AB_Type.h:83-130), then initializes."""
        if representation is not None:
            self.set_representation(representation)
        self.setPeriodicity(*[bool(p) for p in system.periodic])
        self.setNrOfAllMonomers(system.n)
        self.set_coords(system.xyz)
        attrs = np.ascontiguousarray(system.attributes, dtype=np.int32)
        self._call("bfm_set_attributes_bulk", attrs, system.n)
        rows, cols = system.bonds()
        pairs = np.ascontiguousarray(np.stack([rows, cols], axis=1), dtype=np.uint32).reshape(-1)
        self._call("bfm_add_bonds_bulk", pairs, pairs.size // 2)
        self.setLatticeSize(*system.box)
        self.populateLattice()
        forb = system.forbidden
        for dx in range(-4, 4):
            for dy in range(-4, 4):
                for dz in range(-4, 4):
                    idx = (dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)
                    self._L.bfm_set_bond_forbidden(self._h, dx, dy, dz, int(forb[idx]))
        self.set_seed(system.seed if seed is None else seed)
        if mode is not None:
            self.set_mode(mode)
        if initialize:
            self.initialize()
        return self


class Batch:
    """Many initialised updaters on one GPU advanced together (include/bfm.h, bfm_batch_*)."""

    def __init__(self, members, gpu: int = 0, resident: bool = True, cluster: bool = True):
        self._L = _lib.load()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.handle for m in self.members])
        h = C.c_void_p()
        st = self._L.bfm_batch_create(C.byref(h), gpu, arr, len(self.members))
        if st != _lib.BFM_OK:
            _lib.raise_for(st, self._L.bfm_batch_last_error(None).decode())
        self._h = h
        if not resident:
            self._call("bfm_batch_set_resident", 0)
        if not cluster:
            self._call("bfm_batch_set_cluster", 0)

    def _call(self, name, *args):
        st = getattr(self._L, name)(self._h, *args)
        if st != _lib.BFM_OK:
            _lib.raise_for(st, self._L.bfm_batch_last_error(self._h).decode())

    def run(self, n_mcs: int):
        self._call("bfm_batch_run", n_mcs)

    def run_async(self, n_mcs: int):
        self._call("bfm_batch_run_async", n_mcs)

    def set_shape(self, shape: int):
        """Register budget of the grid-phase kernels (0..3, -1 = default); results do not change."""
        self._call("bfm_batch_set_shape", shape)

    def set_block(self, block: int):
        """CTA size of the grid groups' check (128, 256, 512; 0 = default); results do not change."""
        self._call("bfm_batch_set_block", block)

    def set_perform(self, warps: int, group: int):
        """Warps per CTA and per tile of the grid groups' perform (1, 2, 4, 8, group <= warps; 0, 0 =
        default); results do not change."""
        self._call("bfm_batch_set_perform", warps, group)

    def perform_shape(self) -> tuple:
        w, g = C.c_int(), C.c_int()
        self._call("bfm_batch_get_perform", C.byref(w), C.byref(g))
        return w.value, g.value

    def autotune(self, mcs_per_trial: int = 10) -> dict:
        """Times the configurations in three stages (the resident / cluster paths on or off; the grid
        check's register budget x CTA size for the best paths; the perform's warps per CTA x per
        tile for the best of those), 1 + mcs_per_trial MCS each, and keeps the fastest. The trials
        advance every member (the results do not depend on the configuration)."""
        cap = 64
        trials = np.zeros(6 * cap, dtype=np.float32)
        shape, paths, best, n = C.c_int(), C.c_int(), C.c_float(), C.c_uint32()
        self._call("bfm_batch_autotune", mcs_per_trial, C.byref(shape), C.byref(paths), C.byref(best), trials,
                   cap, C.byref(n))
        rows = trials[:6 * min(n.value, cap)].reshape(-1, 6)
        t = [{"shape": int(r[0]), "resident": bool(int(r[1]) & 1), "cluster": bool(int(r[1]) & 2),
              "block": int(r[2]), "perform": (int(r[3]), int(r[4])), "ms_per_mcs": float(r[5])} for r in rows]
        bt = min(t, key=lambda q: q["ms_per_mcs"])
        return {"shape": shape.value, "resident": bool(paths.value & 1), "cluster": bool(paths.value & 2),
                "block": bt["block"], "perform": self.perform_shape(), "ms_per_mcs": best.value,
                "mcs_spent": n.value * (1 + mcs_per_trial), "trials": t}

    def set_cluster(self, on: bool):
        """Members too large for one CTA that a cluster of CTAs holds run in the cluster-resident
        kernel (default on); off: they share the grid-phase kernels. Results do not change."""
        self._call("bfm_batch_set_cluster", 1 if on else 0)

    def run_each(self, mcs):
        """Member i advances mcs[i] MCS (0: it idles)."""
        a = np.ascontiguousarray(mcs, dtype=np.int32)
        if a.shape != (len(self.members),):
            raise ValueError("one MCS count per member")
        self._call("bfm_batch_run_each", a)

    def run_timed(self, n_mcs: int) -> float:
        ms = C.c_float()
        self._call("bfm_batch_run_timed", n_mcs, C.byref(ms))
        return ms.value

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._call("bfm_batch_launch_count", C.byref(v))
        return v.value

    def synchronize(self):
        self._call("bfm_batch_synchronize")

    def close(self):
        if getattr(self, "_h", None):
            self._L.bfm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching job server (include/bfm.h, bfm_server_*)."""

    PENDING, RUNNING, DONE, CANCELLED, FAILED = 0, 1, 2, 3, 4

    def __init__(self, gpu: int = 0, budget_bytes: int = 150 << 30, max_jobs: int = 1024):
        self._L = _lib.load()
        h = C.c_void_p()
        st = self._L.bfm_server_create(C.byref(h), gpu, budget_bytes, max_jobs)
        if st != _lib.BFM_OK:
            _lib.raise_for(st, self._L.bfm_server_last_error(None).decode())
        self._h = h
        self._sizes = {}

    def _call(self, name, *args):
        st = getattr(self._L, name)(self._h, *args)
        if st != _lib.BFM_OK:
            _lib.raise_for(st, self._L.bfm_server_last_error(self._h).decode())

    def submit(self, system, n_mcs: int, every: int, seed: int | None = None) -> int:
        """Queues system (a systems.BfmSystem) for n_mcs MCS with observables every `every` MCS."""
        setup = UpdaterGPUScBFM_AB_Type(0)
        setup.load_system(system, seed=seed, initialize=False)
        return self.submit_setup(setup, n_mcs, every, n=system.n)

    def submit_setup(self, setup: "UpdaterGPUScBFM_AB_Type", n_mcs: int, every: int, n: int) -> int:
        job = C.c_uint64()
        self._call("bfm_server_submit", setup.handle, n_mcs, every, C.byref(job))
        self._sizes[job.value] = (n, n_mcs, every)
        return job.value

    @staticmethod
    def estimate_bytes(system) -> int:
        """Device bytes admission charges for a job on `system` (a systems.BfmSystem)."""
        setup = UpdaterGPUScBFM_AB_Type(0)
        setup.load_system(system, initialize=False)
        v = C.c_uint64()
        setup._call("bfm_server_estimate_bytes", C.byref(v))
        setup.close()
        return v.value

    def status(self, job: int) -> int:
        v = C.c_int()
        self._call("bfm_server_status", job, C.byref(v))
        return v.value

    def cancel(self, job: int):
        self._call("bfm_server_cancel", job)

    def wait(self, job: int, timeout: float = 600.0):
        self._call("bfm_server_wait", job, timeout)

    def result(self, job: int):
        """(final positions (n, 3), samples (n_samples, 5 n_mol + 513) int64, latency in s)."""
        n, n_mcs, every = self._sizes[job]
        xyz = np.zeros((n, 3), dtype=np.int32)
        ns = C.c_uint32()
        lat = C.c_double()
        words = C.c_uint64()
        self._call("bfm_server_sample_words", job, C.byref(words))
        samples = np.zeros(words.value, dtype=np.int64)
        self._call("bfm_server_result", job, xyz.ctypes.data, n, samples.ctypes.data, samples.size, C.byref(ns),
                   C.byref(lat))
        return xyz, samples.reshape(ns.value, -1), lat.value

    def stats(self) -> dict:
        out = np.zeros(8, dtype=np.float64)
        self._call("bfm_server_stats", out)
        keys = ["completed", "failed", "moves", "p50_s", "p99_s", "mean_s", "resident_bytes", "elapsed_s"]
        return dict(zip(keys, out.tolist()))

    def job_times(self, job: int) -> tuple:
        """(arrival, admission, completion) in seconds since the server started; -1 = not yet."""
        out = np.zeros(3, dtype=np.float64)
        self._call("bfm_server_job_times", job, out)
        return tuple(out.tolist())

    def inject_fault(self, kind: int = 1):
        self._call("bfm_server_inject_fault", kind)

    def close(self):
        if getattr(self, "_h", None):
            self._L.bfm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
