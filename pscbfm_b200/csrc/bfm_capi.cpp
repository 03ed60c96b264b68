// C-ABI of the engine (include/bfm.h): exceptions of the C++ layer become status codes.

#include "../../include/bfm.h"

#include <algorithm>
#include <new>
#include <stdexcept>
#include <string>

#include "bfm_engine.hpp"
#include "bfm_server.hpp"

struct bfm_server {
    bfm::Server s;
    std::string err;
    bfm_server(int gpu, size_t budget, uint32_t maxJobs) : s(gpu, budget, maxJobs) {}
};

struct bfm_updater {
    bfm::Updater u;
    std::string err;
    explicit bfm_updater(int gpu) : u(gpu) {}
};

struct bfm_batch {
    bfm::Batch b;
    std::string err;
    bfm_batch(int gpu, bfm::Updater* const* m, uint32_t n) : b(gpu, m, n) {}
};

namespace {

thread_local std::string gErr;

template <typename F>
int guarded(std::string* sink, F&& f)
{
    try {
        f();
        return BFM_OK;
    } catch (bfm::CudaError const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_CUDA;
    } catch (std::out_of_range const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_OUT_OF_RANGE;
    } catch (std::invalid_argument const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_INVALID_ARGUMENT;
    } catch (std::bad_alloc const&) {
        (sink ? *sink : gErr) = "host allocation failed";
        return BFM_ERR_RUNTIME;
    } catch (bfm::BudgetError const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_BUDGET;
    } catch (bfm::BusyError const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_BUSY;
    } catch (std::exception const& e) {
        (sink ? *sink : gErr) = e.what();
        return BFM_ERR_RUNTIME;
    }
}

#define BFM_CALL(h, ...)                                          \
    do {                                                          \
        if (!(h)) {                                               \
            gErr = "null handle";                                 \
            return BFM_ERR_NULL_HANDLE;                           \
        }                                                         \
        return guarded(&(h)->err, [&] { __VA_ARGS__; });          \
    } while (0)

}  // namespace

extern "C" {

const char* bfm_last_error(bfm_handle h) { return h ? h->err.c_str() : gErr.c_str(); }

int bfm_create(bfm_handle* out, int gpu)
{
    if (!out) {
        gErr = "null output pointer";
        return BFM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return guarded(nullptr, [&] { *out = new bfm_updater(gpu); });
}

int bfm_destroy(bfm_handle h)
{
    if (!h) return BFM_OK;
    delete h;
    return BFM_OK;
}

int bfm_set_gpu(bfm_handle h, int gpu) { BFM_CALL(h, h->u.setGpu(gpu)); }
int bfm_cleanup(bfm_handle h) { BFM_CALL(h, h->u.cleanup()); }
int bfm_set_periodicity(bfm_handle h, int px, int py, int pz) { BFM_CALL(h, h->u.setPeriodicity(px, py, pz)); }
int bfm_set_n_monomers(bfm_handle h, uint32_t n) { BFM_CALL(h, h->u.setNrOfAllMonomers(n)); }
int bfm_set_attribute(bfm_handle h, uint32_t i, int32_t a) { BFM_CALL(h, h->u.setAttribute(i, a)); }
int bfm_set_coords(bfm_handle h, uint32_t i, int32_t x, int32_t y, int32_t z)
{
    BFM_CALL(h, h->u.setMonomerCoordinates(i, x, y, z));
}
int bfm_set_coords_bulk(bfm_handle h, const int32_t* xyz, uint32_t n)
{
    BFM_CALL(h, {
        if (!xyz) throw std::invalid_argument("[bfm_set_coords_bulk] null buffer");
        h->u.setCoordinates(xyz, n);
    });
}
int bfm_add_bond(bfm_handle h, uint32_t a, uint32_t b) { BFM_CALL(h, h->u.setConnectivity(a, b)); }
int bfm_add_bonds_bulk(bfm_handle h, const uint32_t* pairs, uint32_t n)
{
    BFM_CALL(h, {
        if (!pairs && n) throw std::invalid_argument("[bfm_add_bonds_bulk] null buffer");
        for (uint32_t k = 0; k < n; ++k) h->u.setConnectivity(pairs[2 * k], pairs[2 * k + 1]);
    });
}
int bfm_set_attributes_bulk(bfm_handle h, const int32_t* a, uint32_t n)
{
    BFM_CALL(h, {
        if (!a && n) throw std::invalid_argument("[bfm_set_attributes_bulk] null buffer");
        for (uint32_t i = 0; i < n; ++i) h->u.setAttribute(i, a[i]);
    });
}
int bfm_set_box(bfm_handle h, uint32_t bx, uint32_t by, uint32_t bz) { BFM_CALL(h, h->u.setLatticeSize(bx, by, bz)); }
int bfm_set_bond_forbidden(bfm_handle h, int dx, int dy, int dz, int f)
{
    BFM_CALL(h, h->u.copyBondSet(dx, dy, dz, f != 0));
}
int bfm_set_standard_bond_set(bfm_handle h)
{
    BFM_CALL(h, {
        // every sign/permutation of (2,0,0) (2,1,0) (2,1,1) (2,2,1) (3,0,0) (3,1,0)
        static int const base[6][3] = {{2, 0, 0}, {2, 1, 0}, {2, 1, 1}, {2, 2, 1}, {3, 0, 0}, {3, 1, 0}};
        static int const perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        for (int dx = -4; dx < 4; ++dx)
            for (int dy = -4; dy < 4; ++dy)
                for (int dz = -4; dz < 4; ++dz) h->u.copyBondSet(dx, dy, dz, true);
        for (auto const& b : base)
            for (auto const& p : perm)
                for (int s = 0; s < 8; ++s) {
                    int const v[3] = {b[p[0]] * ((s & 1) ? -1 : 1), b[p[1]] * ((s & 2) ? -1 : 1),
                                      b[p[2]] * ((s & 4) ? -1 : 1)};
                    h->u.copyBondSet(v[0], v[1], v[2], false);
                }
    });
}
int bfm_populate_lattice(bfm_handle h) { BFM_CALL(h, h->u.populateLattice()); }
int bfm_set_seed(bfm_handle h, uint64_t seed) { BFM_CALL(h, h->u.setDrawCounter(seed)); }
int bfm_set_substep(bfm_handle h, uint64_t substep) { BFM_CALL(h, h->u.setSubStep(substep)); }
int bfm_get_substep(bfm_handle h, uint64_t* substep)
{
    BFM_CALL(h, {
        if (!substep) throw std::invalid_argument("[bfm_get_substep] null output");
        *substep = h->u.subStep();
    });
}
int bfm_set_draw_callback(bfm_handle h, bfm_draw_fn fn, void* ctx) { BFM_CALL(h, h->u.setDrawCallback(fn, ctx)); }
int bfm_set_mode(bfm_handle h, int mode) { BFM_CALL(h, h->u.setMode(mode)); }
int bfm_set_representation(bfm_handle h, int r) { BFM_CALL(h, h->u.setRepresentation(r)); }
int bfm_get_representation(bfm_handle h, int* out)
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_get_representation] null output");
        *out = (int)h->u.codeMode();
    });
}
int bfm_set_grid_block(bfm_handle h, int block) { BFM_CALL(h, h->u.setGridBlock(block)); }
int bfm_set_perform(bfm_handle h, int warps, int group) { BFM_CALL(h, h->u.setPerformShape(warps, group)); }
int bfm_initialize(bfm_handle h) { BFM_CALL(h, h->u.initialize()); }
int bfm_run(bfm_handle h, int32_t n) { BFM_CALL(h, h->u.runSimulationOnGPU(n)); }
int bfm_run_async(bfm_handle h, int32_t n) { BFM_CALL(h, h->u.run(n)); }
int bfm_inject_barrier_stall(bfm_handle h) { BFM_CALL(h, h->u.injectBarrierStall()); }
int bfm_get_path(bfm_handle h, int* mode)
{
    BFM_CALL(h, {
        if (!mode) throw std::invalid_argument("[bfm_get_path] null output");
        *mode = h->u.path();
    });
}
int bfm_synchronize(bfm_handle h) { BFM_CALL(h, h->u.synchronize()); }
int bfm_get_coord(bfm_handle h, uint32_t i, int axis, int32_t* out)
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_get_coord] null output");
        *out = h->u.getMonomerPosition(i, axis);
    });
}
int bfm_get_coords_bulk(bfm_handle h, int32_t* xyz, uint32_t n)
{
    BFM_CALL(h, {
        if (!xyz) throw std::invalid_argument("[bfm_get_coords_bulk] null buffer");
        h->u.getCoordinates(xyz, n);
    });
}
int bfm_n_colors(bfm_handle h, uint32_t* nColors, uint32_t* sizes, uint32_t capacity)
{
    BFM_CALL(h, {
        auto const g = h->u.groupSizes();
        if (nColors) *nColors = (uint32_t)g.size();
        if (sizes)
            for (uint32_t c = 0; c < g.size() && c < capacity; ++c) sizes[c] = g[c];
    });
}
int bfm_get_stats(bfm_handle h, uint64_t out[4])
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_get_stats] null output");
        h->u.stats(out);
    });
}
int bfm_stats_enqueue(bfm_handle h, uint64_t* ticket)
{
    BFM_CALL(h, {
        if (!ticket) throw std::invalid_argument("[bfm_stats_enqueue] null output");
        *ticket = h->u.statsEnqueue();
    });
}
int bfm_stats_wait(bfm_handle h, uint64_t ticket, uint64_t out[4])
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_stats_wait] null output");
        h->u.statsWait(ticket, out);
    });
}
int bfm_validate(bfm_handle h) { BFM_CALL(h, h->u.validate()); }
int bfm_device_bytes(bfm_handle h, uint64_t* out)
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_device_bytes] null output");
        *out = h->u.deviceBytes();
    });
}

int bfm_n_molecules(bfm_handle h, uint32_t* n)
{
    BFM_CALL(h, {
        if (!n) throw std::invalid_argument("[bfm_n_molecules] null output");
        h->u.moleculeSizes();   // requires initialize
        *n = h->u.nMolecules();
    });
}
int bfm_molecule_sizes(bfm_handle h, uint32_t* sizes, uint32_t cap)
{
    BFM_CALL(h, {
        auto const m = h->u.moleculeSizes();
        if (!sizes && cap) throw std::invalid_argument("[bfm_molecule_sizes] null output");
        for (uint32_t i = 0; i < m.size() && i < cap; ++i) sizes[i] = m[i];
    });
}
int bfm_observables(bfm_handle h, int64_t* out, uint64_t cap)
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_observables] null output");
        h->u.moleculeSizes();
        if (cap < bfm::obs_words(h->u.nMolecules()))
            throw std::invalid_argument("[bfm_observables] output holds fewer than 5*n_mol+513 words");
        h->u.observables(reinterpret_cast<long long*>(out));
    });
}
int bfm_reset_msd_reference(bfm_handle h) { BFM_CALL(h, h->u.resetReference()); }

int bfm_run_timed(bfm_handle h, int32_t n, float* ms)
{
    BFM_CALL(h, {
        if (!ms) throw std::invalid_argument("[bfm_run_timed] null output");
        *ms = h->u.runTimed(n);
    });
}
int bfm_time_kernels(bfm_handle h, int32_t n, double out[4])
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_time_kernels] null output");
        h->u.timeKernels(n, out);
    });
}
int bfm_launch_count(bfm_handle h, uint64_t* out)
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_launch_count] null output");
        *out = h->u.launches();
    });
}
int bfm_transfer_bytes(bfm_handle h, uint64_t out[2])
{
    BFM_CALL(h, {
        if (!out) throw std::invalid_argument("[bfm_transfer_bytes] null output");
        out[0] = h->u.h2dBytes();
        out[1] = h->u.d2hBytes();
    });
}

// ---------------------------------------------------------------- server

const char* bfm_server_last_error(bfm_server_handle s) { return s ? s->err.c_str() : gErr.c_str(); }

int bfm_server_create(bfm_server_handle* out, int gpu, uint64_t budget, uint32_t maxJobs)
{
    if (!out) {
        gErr = "null output pointer";
        return BFM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return guarded(nullptr, [&] { *out = new bfm_server(gpu, (size_t)budget, maxJobs); });
}

int bfm_server_destroy(bfm_server_handle s)
{
    if (!s) return BFM_OK;
    delete s;
    return BFM_OK;
}

int bfm_server_submit(bfm_server_handle s, bfm_handle setup, int32_t nMcs, int32_t every, uint64_t* job)
{
    BFM_CALL(s, {
        if (!setup || !job) throw std::invalid_argument("[bfm_server_submit] null argument");
        *job = s->s.submit(setup->u, nMcs, every);
    });
}
int bfm_server_estimate_bytes(bfm_handle setup, uint64_t* bytes)
{
    BFM_CALL(setup, {
        if (!bytes) throw std::invalid_argument("[bfm_server_estimate_bytes] null output");
        setup->u.checkSetup();
        *bytes = bfm::Server::estimateBytes(setup->u);
    });
}
int bfm_server_status(bfm_server_handle s, uint64_t job, int* state)
{
    BFM_CALL(s, {
        if (!state) throw std::invalid_argument("[bfm_server_status] null output");
        *state = s->s.status(job);
    });
}
int bfm_server_cancel(bfm_server_handle s, uint64_t job) { BFM_CALL(s, s->s.cancel(job)); }
int bfm_server_wait(bfm_server_handle s, uint64_t job, double timeout)
{
    BFM_CALL(s, {
        if (!s->s.wait(job, timeout)) throw bfm::BusyError("[bfm_server_wait] timed out");
    });
}
int bfm_server_result(bfm_server_handle s, uint64_t job, int32_t* xyz, uint32_t n, int64_t* samples, uint64_t cap,
                      uint32_t* nSamples, double* latency)
{
    BFM_CALL(s, s->s.result(job, xyz, n, reinterpret_cast<long long*>(samples), cap, nSamples, latency));
}
int bfm_server_sample_words(bfm_server_handle s, uint64_t job, uint64_t* words)
{
    BFM_CALL(s, {
        if (!words) throw std::invalid_argument("[bfm_server_sample_words] null output");
        *words = s->s.sampleWords(job);
    });
}
int bfm_server_job_times(bfm_server_handle s, uint64_t job, double out[3])
{
    BFM_CALL(s, {
        if (!out) throw std::invalid_argument("[bfm_server_job_times] null output");
        s->s.jobTimes(job, out);
    });
}
int bfm_server_stats(bfm_server_handle s, double out[8])
{
    BFM_CALL(s, {
        if (!out) throw std::invalid_argument("[bfm_server_stats] null output");
        s->s.stats(out);
    });
}
int bfm_server_inject_fault(bfm_server_handle s, int kind) { BFM_CALL(s, s->s.injectFault(kind)); }

// ---------------------------------------------------------------- host-only helpers

int bfm_color_graph(uint32_t n, const uint32_t* counts, const uint32_t* ids, uint32_t stride, uint8_t* out,
                    uint32_t* nColors)
{
    return guarded(nullptr, [&] {
        if (n == 0) throw std::invalid_argument("[bfm_color_graph] no monomers");
        if (!counts || !ids || !out) throw std::invalid_argument("[bfm_color_graph] null buffer");
        for (uint32_t i = 0; i < n; ++i) {
            if (counts[i] > stride) throw std::invalid_argument("[bfm_color_graph] count exceeds stride");
            for (uint32_t k = 0; k < counts[i]; ++k)
                if (ids[(size_t)i * stride + k] >= n) throw std::out_of_range("[bfm_color_graph] neighbour id out of range");
        }
        auto const c = bfm::colour_bond_graph(n, counts, ids, stride);
        uint32_t nc = 0;
        for (uint32_t i = 0; i < n; ++i) {
            out[i] = c[i];
            if ((uint32_t)c[i] + 1 > nc) nc = c[i] + 1u;
        }
        if (nColors) *nColors = nc;
    });
}

uint32_t bfm_counter_draw(uint64_t seed, uint64_t k) { return bfm::counter_draw(seed, k); }

// ---------------------------------------------------------------- batch

const char* bfm_batch_last_error(bfm_batch_handle b) { return b ? b->err.c_str() : gErr.c_str(); }

int bfm_batch_create(bfm_batch_handle* out, int gpu, const bfm_handle* members, uint32_t n)
{
    if (!out || (!members && n)) {
        gErr = "null argument";
        return BFM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return guarded(nullptr, [&] {
        std::vector<bfm::Updater*> m(n);
        for (uint32_t i = 0; i < n; ++i) {
            if (!members[i]) throw std::invalid_argument("[bfm_batch_create] null member handle");
            m[i] = &members[i]->u;
        }
        *out = new bfm_batch(gpu, m.data(), n);
    });
}

int bfm_batch_destroy(bfm_batch_handle b)
{
    if (!b) return BFM_OK;
    delete b;
    return BFM_OK;
}

int bfm_batch_run(bfm_batch_handle b, int32_t n)
{
    BFM_CALL(b, {
        b->b.run(n);
        b->b.synchronize();
    });
}
int bfm_batch_set_shape(bfm_batch_handle b, int shape) { BFM_CALL(b, b->b.setShape(shape)); }
int bfm_batch_set_block(bfm_batch_handle b, int block) { BFM_CALL(b, b->b.setBlock(block)); }
int bfm_batch_set_perform(bfm_batch_handle b, int warps, int group) { BFM_CALL(b, b->b.setPerformShape(warps, group)); }
int bfm_batch_get_perform(bfm_batch_handle b, int* warps, int* group)
{
    BFM_CALL(b, {
        if (warps) *warps = b->b.performWarps();
        if (group) *group = b->b.performGroup();
    });
}
int bfm_batch_autotune(bfm_batch_handle b, int32_t mcsPerTrial, int* shape, int* paths, float* msPerMcs,
                       float* trials, uint32_t capacity, uint32_t* nTrials)
{
    BFM_CALL(b, {
        auto const t = b->b.autotune(mcsPerTrial);
        b->b.synchronize();
        if (shape) *shape = b->b.shape();
        if (paths) *paths = (b->b.residentEnabled() ? 1 : 0) | (b->b.clusterEnabled() ? 2 : 0);
        if (msPerMcs) {
            float best = t.front().msPerMcs;
            for (auto const& x : t) best = std::min(best, x.msPerMcs);
            *msPerMcs = best;
        }
        if (trials)
            for (uint32_t i = 0; i < (uint32_t)t.size() && i < capacity; ++i) {
                float* r = trials + 6 * i;
                r[0] = (float)t[i].shape;
                r[1] = (float)((t[i].resident ? 1 : 0) | (t[i].cluster ? 2 : 0));
                r[2] = (float)t[i].block;
                r[3] = (float)t[i].perfWarps;
                r[4] = (float)t[i].perfGroup;
                r[5] = t[i].msPerMcs;
            }
        if (nTrials) *nTrials = (uint32_t)t.size();
    });
}
int bfm_batch_run_each(bfm_batch_handle b, const int32_t* mcs)
{
    BFM_CALL(b, {
        if (!mcs) throw std::invalid_argument("[bfm_batch_run_each] null MCS array");
        b->b.run(mcs);
        b->b.synchronize();
    });
}
int bfm_batch_run_async(bfm_batch_handle b, int32_t n) { BFM_CALL(b, b->b.run(n)); }
int bfm_batch_run_timed(bfm_batch_handle b, int32_t n, float* ms)
{
    BFM_CALL(b, {
        if (!ms) throw std::invalid_argument("[bfm_batch_run_timed] null output");
        *ms = b->b.runTimed(n);
    });
}
int bfm_batch_synchronize(bfm_batch_handle b) { BFM_CALL(b, b->b.synchronize()); }
int bfm_batch_launch_count(bfm_batch_handle b, uint64_t* out)
{
    BFM_CALL(b, {
        if (!out) throw std::invalid_argument("[bfm_batch_launch_count] null output");
        *out = b->b.launches();
    });
}
int bfm_batch_set_resident(bfm_batch_handle b, int on) { BFM_CALL(b, b->b.setResidentEnabled(on != 0)); }
int bfm_batch_set_cluster(bfm_batch_handle b, int on) { BFM_CALL(b, b->b.setClusterEnabled(on != 0)); }

}  // extern "C"
