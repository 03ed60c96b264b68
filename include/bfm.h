/*
 * bfm.h — C-ABI of the B200 BFM sweep engine (libbfm.so).
 *
 * Drop-in for pscbfm's GPU updater UpdaterGPUScBFM_AB_Type
 * (reference: src/pscbfm/UpdaterGPUScBFM_AB_Type.h:316-358). Every entry point returns a status
 * (BFM_OK or one of the error codes below) instead of throwing; bfm_last_error() returns the
 * message the reference would have put into its exception. Plain pointers and sizes only.
 *
 * Ownership: the engine copies every input into its own host and device buffers; callers keep
 * ownership of what they pass. Handles are independent (no global device state); one handle
 * must not be used from two threads at once, distinct handles may.
 *
 * Draw stream: each sub-step draws a colour (draw % nColors) and a 32-bit seed, in that order
 * (src/pscbfm/CRITICAL.cu:509-510). The default stream is counter-based: draw k of a system with
 * seed S is the upper 32 bits of SplitMix64(SplitMix64(S) + (k+1) * 0x9E3779B97F4A7C15), sub-step
 * t uses draws 2t and 2t+1. An external generator (e.g. LeMonADE's r250) can be plugged in with
 * bfm_set_draw_callback.
 */
#ifndef BFM_H
#define BFM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define BFM_OK 0
#define BFM_ERR_INVALID_ARGUMENT 1 /* reference: std::invalid_argument */
#define BFM_ERR_RUNTIME 2          /* reference: std::runtime_error */
#define BFM_ERR_CUDA 3             /* reference: CUDA_ERROR -> exit(EXIT_FAILURE), cudacommon.hpp:31-46 */
#define BFM_ERR_OUT_OF_RANGE 4     /* reference: std::out_of_range from vector::at */
#define BFM_ERR_NULL_HANDLE 5
#define BFM_ERR_BUDGET 6           /* server admission: job larger than the memory budget */
#define BFM_ERR_BUSY 7             /* server: result not ready yet */

/* engine paths (bfm_set_mode) */
#define BFM_MODE_AUTO 0     /* resident for small systems (largest colour group <= 2048 and fits one CTA),
                               cluster where a cluster's shared memory holds the system with at
                               most 48 chunks of 32 slots per CTA and colour (one per warp where a
                               cluster of up to 16 CTAs allows), persistent up to about
                               three 512-monomer tiles per SM (bond codes), else graph */
#define BFM_MODE_LAUNCH 1   /* check + perform launch per sub-step (the reference's structure) */
#define BFM_MODE_GRAPH 2    /* the same launches captured into CUDA graphs */
#define BFM_MODE_RESIDENT 3 /* one CTA per system, lattice in shared memory (box <= 64^3) */
#define BFM_MODE_PERSISTENT 4 /* bond codes: one cooperative launch runs a whole chunk of sub-steps,
                                 grid barriers between the phases (gather systems use GRAPH) */
#define BFM_MODE_CLUSTER 5    /* bond codes: one thread-block cluster (2-16 CTAs) holds the system's
                                 lattice and state in its shared memory for a whole chunk of
                                 sub-steps (systems too large for one CTA, up to about 200 KB x 16) */

typedef struct bfm_updater* bfm_handle;
typedef struct bfm_batch* bfm_batch_handle;
typedef uint32_t (*bfm_draw_fn)(void* ctx);

/* Last error message of a handle (NULL handle: of the last failed call without a handle on this
 * thread). Valid until the next call on that handle. */
const char* bfm_last_error(bfm_handle h);

/* ------------------------------------------------------------------ life cycle */
/* Constructor + setGpu (UpdaterGPUScBFM_AB_Type.cu:416-450, :472-487). */
int bfm_create(bfm_handle* out, int gpu);
/* Destructor (UpdaterGPUScBFM_AB_Type.cu:467-470). */
int bfm_destroy(bfm_handle h);
/* setGpu (UpdaterGPUScBFM_AB_Type.cu:472-487); invalid_argument if the GPU does not exist. */
int bfm_set_gpu(bfm_handle h, int gpu);
/* cleanup (UpdaterGPUScBFM_AB_Type.cu:995-1001): frees the device state; the handle returns to
 * its freshly created state so the setter sequence can be repeated. */
int bfm_cleanup(bfm_handle h);

/* ------------------------------------------------------------------ setters */
/* setPeriodicity (UpdaterGPUScBFM_AB_Type.cu:728-753), before bfm_initialize. The reference's
 * default build takes fully periodic boxes and its NONPERIODICITY build fully non-periodic ones;
 * here each axis chooses. Along an axis without periodicity, corners must lie in [0, L-2] and a move
 * that would leave that range is rejected (CRITICAL.cu:334-341). */
int bfm_set_periodicity(bfm_handle h, int px, int py, int pz);
/* setNrOfAllMonomers (UpdaterGPUScBFM_AB_Type.cu:699-726); runtime error if already set. */
int bfm_set_n_monomers(bfm_handle h, uint32_t n);
/* setAttribute (UpdaterGPUScBFM_AB_Type.cu:755-758). */
int bfm_set_attribute(bfm_handle h, uint32_t i, int32_t attribute);
/* Bulk form of setAttribute for monomers 0..n-1. */
int bfm_set_attributes_bulk(bfm_handle h, const int32_t* attributes, uint32_t n);
/* setMonomerCoordinates (UpdaterGPUScBFM_AB_Type.cu:760-771), lower-left-front corner, unfolded. */
int bfm_set_coords(bfm_handle h, uint32_t i, int32_t x, int32_t y, int32_t z);
/* Bulk form of setMonomerCoordinates: xyz[3*i+a]. After bfm_initialize it uploads the new
 * positions and rebuilds the occupancy lattice on the device. */
int bfm_set_coords_bulk(bfm_handle h, const int32_t* xyz, uint32_t n);
/* setConnectivity (UpdaterGPUScBFM_AB_Type.cu:777-795): directed, call once per direction.
 * At most 16 neighbours per monomer (the reference's compile-time MAX_CONNECTIVITY is 4). */
int bfm_add_bond(bfm_handle h, uint32_t a, uint32_t b);
/* Bulk form: pairs[2*k] -> pairs[2*k+1] for k < n_pairs, in order (same as n_pairs calls). */
int bfm_add_bonds_bulk(bfm_handle h, const uint32_t* pairs, uint32_t n_pairs);
/* setLatticeSize (UpdaterGPUScBFM_AB_Type.cu:797-848): 4..1024 per side, a power of two along a
 * periodic axis (the reference's rule for every axis); along an axis without periodicity any side
 * (the lattice there is the next power of two; nothing wraps). A non-power-of-two side on an axis
 * that is periodic when this or bfm_set_periodicity is called is BFM_ERR_RUNTIME. */
int bfm_set_box(bfm_handle h, uint32_t bx, uint32_t by, uint32_t bz);
/* copyBondSet (UpdaterGPUScBFM_AB_Type.cu:693-697): entry (dx&7)|(dy&7)<<3|(dz&7)<<6 of the
 * 512-entry table; everything starts forbidden. */
int bfm_set_bond_forbidden(bfm_handle h, int dx, int dy, int dz, int forbidden);
/* Convenience: load the standard 108-vector set (GPUScBFM_AB_Type.h:120-127 with LeMonADE's
 * default bond set). */
int bfm_set_standard_bond_set(bfm_handle h);
/* populateLattice (UpdaterGPUScBFM_AB_Type.cu:850-872). */
int bfm_populate_lattice(bfm_handle h);
/* Draw stream (replaces the RandomNumberGenerators member, UpdaterGPUScBFM_AB_Type.h:131). */
int bfm_set_seed(bfm_handle h, uint64_t seed);
/* Position of the counter draw stream: the sub-steps drawn so far (0 after bfm_initialize). A run
 * resumed from a checkpoint sets the saved position after bfm_initialize and continues bit-exactly.
 * No counterpart in the reference, whose generator state is not saved. */
int bfm_set_substep(bfm_handle h, uint64_t substep);
int bfm_get_substep(bfm_handle h, uint64_t* substep);
int bfm_set_draw_callback(bfm_handle h, bfm_draw_fn fn, void* ctx);
/* Engine path, BFM_MODE_*. */
int bfm_set_mode(bfm_handle h, int mode);
/* CTA size of the check on this handle's grid paths (bond codes): 128, 256 or 512 threads over the
 * same 512-monomer tile (0: the default, 256); results do not change. No reference counterpart:
 * the reference's runSimulationOnGPU times block sizes itself when built with
 * AUTO_CONFIGURE_BEST_SETTINGS_FOR_PSCBFM_ALGORITHM (CRITICAL.cu:445-487). */
int bfm_set_grid_block(bfm_handle h, int block);
/* Warps per CTA and warps per tile of the perform on this handle's grid paths (bond codes): each 1,
 * 2, 4 or 8, the second at most the first (0, 0: the default, 4 and 4); results do not change. No
 * reference counterpart (the reference's perform runs one thread per monomer of the colour). */
int bfm_set_perform(bfm_handle h, int warps, int group);
/* The path the next run takes (after bfm_initialize): the mode set by bfm_set_mode with
 * BFM_MODE_AUTO resolved, and a mode the system cannot use replaced by BFM_MODE_GRAPH. */
int bfm_get_path(bfm_handle h, int* mode);
/* Fault injection for tests (no counterpart in the reference): the next BFM_MODE_PERSISTENT launch
 * of this handle runs as a cooperative grid (never as one cluster, whose barriers are in hardware)
 * and starts its grid-barrier arrival count where no barrier can complete, so every
 * CTA's wait runs out at its time limit (2 s) and the run reports the timeout (BFM_ERR_CUDA).
 * Nothing faults on the GPU and the device stays usable; this system's state is not. */
int bfm_inject_barrier_stall(bfm_handle h);
/* Device representation of the bonds, chosen before bfm_initialize: BFM_REPR_AUTO (bond codes —
 * each monomer keeps the table indices of its bonds, updated exactly when it or a neighbour moves
 * — when every bond is listed in both directions and no monomer has more than 6; otherwise the
 * neighbours' positions are gathered like the reference does) or BFM_REPR_GATHER. Results are
 * identical; only speed differs. */
#define BFM_REPR_AUTO 0
#define BFM_REPR_GATHER 1
int bfm_set_representation(bfm_handle h, int repr);
/* The representation initialize chose: 0 gather, 1 bond codes (32-bit), 2 bond codes (64-bit). */
int bfm_get_representation(bfm_handle h, int* out);

/* ------------------------------------------------------------------ simulation */
/* initialize (UpdaterGPUScBFM_AB_Type.cu:490-690): bond-set check (exactly 108 allowed),
 * colouring, per-colour groups, device upload. */
int bfm_initialize(bfm_handle h);
/* runSimulationOnGPU (CRITICAL.cu:414-698): nMCS Monte Carlo steps; returns when done. */
int bfm_run(bfm_handle h, int32_t n_mcs);
/* The same, returning as soon as the work is queued on the handle's stream. */
int bfm_run_async(bfm_handle h, int32_t n_mcs);
int bfm_synchronize(bfm_handle h);

/* ------------------------------------------------------------------ read back */
/* getMonomerPositionIn{X,Y,Z} (UpdaterGPUScBFM_AB_Type.cu:773-775); axis 0,1,2. */
int bfm_get_coord(bfm_handle h, uint32_t i, int axis, int32_t* out);
/* All positions, xyz[3*i+a], original monomer order. */
int bfm_get_coords_bulk(bfm_handle h, int32_t* xyz, uint32_t n);
/* Number of colour groups (mnElementsInGroup.size(), UpdaterGPUScBFM_AB_Type.cu:559-565) and
 * their sizes (sizes may be NULL). */
int bfm_n_colors(bfm_handle h, uint32_t* n_colors, uint32_t* sizes, uint32_t capacity);
/* Counters since initialize: attempted moves, tentatively accepted (check passed), accepted,
 * MCS done. */
int bfm_get_stats(bfm_handle h, uint64_t out[4]);
/* The same counters without waiting for later work (no reference counterpart): bfm_stats_enqueue
 * returns a ticket for the counters as the work queued so far on the handle leaves them;
 * bfm_stats_wait waits for their copy only, while work queued after it keeps running, and writes
 * the counters as they stood then. After a graph-path run (bond codes) the copy comes from the
 * snapshot the next run's first kernel takes, so the sweep's stream carries no extra kernel; when
 * no such run follows, the wait (or any other work on the handle) reads the counters directly.
 * The last 8 tickets of a handle stay valid; an older or unknown ticket is
 * BFM_ERR_INVALID_ARGUMENT. */
int bfm_stats_enqueue(bfm_handle h, uint64_t* ticket);
int bfm_stats_wait(bfm_handle h, uint64_t ticket, uint64_t out[4]);
/* checkSystem (UpdaterGPUScBFM_AB_Type.cu:882-986): excluded volume and bond set on the host. */
int bfm_validate(bfm_handle h);
/* Device bytes held by the handle. */
int bfm_device_bytes(bfm_handle h, uint64_t* out);

/* ------------------------------------------------------------------ observables (no reference counterpart) */
/* Molecules are the connected components of the bonds, numbered by their lowest monomer id. */
int bfm_n_molecules(bfm_handle h, uint32_t* n_mol);
int bfm_molecule_sizes(bfm_handle h, uint32_t* sizes, uint32_t capacity);
/* Exact int64 observables of the current configuration, 5*n_mol + 513 words:
 *   [4m .. 4m+3]      molecule m: sum x, sum y, sum z, sum (x^2+y^2+z^2)  (Rg^2 = S2/n - |S1|^2/n^2)
 *   [4 n_mol + m]     molecule m: |r_last - r_first|^2 (lowest and highest monomer id)
 *   [5 n_mol + idx]   bond-vector histogram by table index (dx&7)|(dy&7)<<3|(dz&7)<<6, every listed bond
 *   [5 n_mol + 512]   sum over monomers of |r - r_ref|^2 (r_ref: positions at initialize or last reset) */
int bfm_observables(bfm_handle h, int64_t* out, uint64_t capacity_words);
/* Makes the current positions the reference of the displacement sum. */
int bfm_reset_msd_reference(bfm_handle h);

/* ------------------------------------------------------------------ measurement (no reference counterpart) */
/* bfm_run bracketed by CUDA events on the handle's stream; *ms = device time of the n_mcs MCS. */
int bfm_run_timed(bfm_handle h, int32_t n_mcs, float* ms);
/* Runs n_mcs MCS on the grid-phase kernels one launch at a time, each bracketed by CUDA events:
 * out = {check ms total, perform ms total, check launches, perform launches}. */
int bfm_time_kernels(bfm_handle h, int32_t n_mcs, double out[4]);
/* Kernels this handle has launched so far (graph replays counted per kernel). */
int bfm_launch_count(bfm_handle h, uint64_t* out);
/* Bytes the run and read-back calls of this handle have copied so far: out[0] host -> device (step
 * entries; with the counter draw stream on the graph path only the first entry of a chain, the
 * device makes the rest), out[1] device -> host (positions, move counters). Set-up uploads are not
 * counted. */
int bfm_transfer_bytes(bfm_handle h, uint64_t out[2]);
/* Device probes for the sweep's latency model, on GPU gpu: out = {L2 hit latency in ns (dependent
 * loads of a random cycle through 8 MB, one per 128-byte line), L2 read bandwidth in GB/s (32 MB
 * read 20 times by every SM), period in us of back-to-back empty kernels of 1024 x 256 threads in a
 * captured graph, SM count}. Allocates and frees about 40 MB; synchronises the device's work on
 * its own stream only. */
int bfm_probe_device(int gpu, double out[4]);

/* ------------------------------------------------------------------ host-only helpers (no GPU needed) */
/* The colouring step of initialize (graphColoring.tpp:77-293 with uniform rebalancing,
 * UpdaterGPUScBFM_AB_Type.cu:549-555): colours_out[i] for monomer i; returns the status and
 * writes the colour count. ids[i*stride + k] is neighbour k of monomer i. */
int bfm_color_graph(uint32_t n, const uint32_t* counts, const uint32_t* ids, uint32_t stride,
                    uint8_t* colours_out, uint32_t* n_colors);
/* Draw k of the counter stream with the given seed. */
uint32_t bfm_counter_draw(uint64_t seed, uint64_t k);

/* ------------------------------------------------------------------ batch (no reference counterpart) */
/* Advances many initialised handles on one GPU together; each keeps its own draw stream, so its
 * trajectory equals a run alone. Handles stay owned by the caller and must outlive the batch. */
int bfm_batch_create(bfm_batch_handle* out, int gpu, const bfm_handle* members, uint32_t n);
int bfm_batch_destroy(bfm_batch_handle b);
int bfm_batch_run(bfm_batch_handle b, int32_t n_mcs);        /* returns when done */
int bfm_batch_run_async(bfm_batch_handle b, int32_t n_mcs);
/* bfm_batch_run bracketed by CUDA events on the batch stream; *ms = device time. */
int bfm_batch_run_timed(bfm_batch_handle b, int32_t n_mcs, float* ms);
/* Kernels the batch has launched so far (graph replays counted per kernel). */
int bfm_batch_launch_count(bfm_batch_handle b, uint64_t* out);
int bfm_batch_synchronize(bfm_batch_handle b);
/* 0: every system on the grid path; 1 (default): small systems on the resident kernel. */
int bfm_batch_set_resident(bfm_batch_handle b, int on);
/* 1 (default): systems too large for one CTA that a cluster of CTAs holds with at most two chunks
 * of 32 monomers per warp and colour (bond codes; there the cluster-resident kernel of
 * BFM_MODE_CLUSTER beats the grid-phase kernels) run in that kernel while the batch's clusters take
 * at most half of the SMs; 0: they share the grid-phase kernels. */
int bfm_batch_set_cluster(bfm_batch_handle b, int on);
/* Member i advances mcs[i] MCS (0 = it idles); one launch sequence for all, like bfm_batch_run. */
int bfm_batch_run_each(bfm_batch_handle b, const int32_t* mcs);
/* Register budget of the grid-phase kernels, 0..3, or -1 for the default; results do not change. */
int bfm_batch_set_shape(bfm_batch_handle b, int shape);
/* CTA size of the grid groups' check: 128, 256 or 512 threads over the same 512-monomer tile (0:
 * the default, 256); results do not change. */
int bfm_batch_set_block(bfm_batch_handle b, int block);
/* Warps per CTA and per tile of the grid groups' perform, as bfm_set_perform (0, 0: the default). */
int bfm_batch_set_perform(bfm_batch_handle b, int warps, int group);
int bfm_batch_get_perform(bfm_batch_handle b, int* warps, int* group);
/* Autotuner: runs configurations for 1 + mcs_per_trial MCS each, keeps the fastest and reports it
 * (shape, paths, ms per MCS; paths: bit 0 the resident path, bit 1 the cluster path). The trials
 * are ordinary MCS of the run (results do not depend on the configuration): every member advances
 * by n_trials x (1 + mcs_per_trial) MCS. Three stages: the paths (resident / cluster kernels on or
 * off) with the grid kernels' defaults; for the best paths the grid check's register budget
 * (shape) x CTA size (128, 256, 512 threads; the reference sweeps its block size,
 * CRITICAL.cu:445-487); for the best of those the perform's warps per CTA x per tile ((8,4),
 * (4,2), (8,8), (2,2) beside the default (4,4)). The last two stages run only when some member is
 * on the grid-phase kernels. trials (may be NULL) receives up to capacity sextuples (shape, paths,
 * block, perform warps, perform warps per tile, ms per MCS; 0 for a default). */
int bfm_batch_autotune(bfm_batch_handle b, int32_t mcs_per_trial, int* shape, int* paths, float* ms_per_mcs,
                       float* trials, uint32_t capacity, uint32_t* n_trials);
const char* bfm_batch_last_error(bfm_batch_handle b);

/* ------------------------------------------------------------------ server (no reference counterpart) */
/* Continuous batching of jobs "run this system for n_mcs MCS, sample observables every k MCS".
 * A worker thread admits jobs in arrival order while their estimated device bytes fit the budget,
 * sets new jobs up while running ones compute, and advances all running jobs together; a job's
 * result equals running it alone. Job states: */
#define BFM_JOB_PENDING 0
#define BFM_JOB_RUNNING 1
#define BFM_JOB_DONE 2
#define BFM_JOB_CANCELLED 3
#define BFM_JOB_FAILED 4
typedef struct bfm_server* bfm_server_handle;
int bfm_server_create(bfm_server_handle* out, int gpu, uint64_t budget_bytes, uint32_t max_jobs);
/* Stops the worker (running jobs are dropped) and frees everything. */
int bfm_server_destroy(bfm_server_handle s);
/* The job's system is the setter state of `setup` (a handle that has NOT been initialised; it is
 * copied, the caller keeps it). BFM_ERR_BUDGET if the job alone exceeds the budget. */
int bfm_server_submit(bfm_server_handle s, bfm_handle setup, int32_t n_mcs, int32_t sample_every, uint64_t* job);
/* The device bytes admission charges for a job built from `setup` (not initialised). */
int bfm_server_estimate_bytes(bfm_handle setup, uint64_t* bytes);
int bfm_server_status(bfm_server_handle s, uint64_t job, int* state);
int bfm_server_cancel(bfm_server_handle s, uint64_t job);
/* Waits up to timeout_s for a final state; BFM_ERR_BUSY on timeout. */
int bfm_server_wait(bfm_server_handle s, uint64_t job, double timeout_s);
/* Final positions (n monomers, may be NULL), the observable samples (ceil(n_mcs/k) records of
 * 5*n_mol+513 int64 words, may be NULL) and the latency from submit to completion.
 * BFM_ERR_BUSY if the job has not finished. */
int bfm_server_result(bfm_server_handle s, uint64_t job, int32_t* xyz, uint32_t n, int64_t* samples,
                      uint64_t capacity_words, uint32_t* n_samples, double* latency_s);
/* Total int64 words of a finished job's samples (n_samples x (5*n_mol+513)); BFM_ERR_BUSY before. */
int bfm_server_sample_words(bfm_server_handle s, uint64_t job, uint64_t* words);
/* out = {arrival, admission, completion} in seconds since bfm_server_create; a time not reached
 * yet is -1. */
int bfm_server_job_times(bfm_server_handle s, uint64_t job, double out[3]);
/* out = {completed, failed, attempted moves of completed jobs, p50 latency s, p99 latency s,
 *        mean latency s, resident device bytes, seconds since create} */
int bfm_server_stats(bfm_server_handle s, double out[8]);
/* Test hook: kind 1 makes the worker thread throw at its next loop (simulated worker death). */
int bfm_server_inject_fault(bfm_server_handle s, int kind);
const char* bfm_server_last_error(bfm_server_handle s);

/* ------------------------------------------------------------------ sweep without allocation */
/* No counterpart in the reference. For callers that must not have the library allocate device
 * memory: programs that reserved the GPU's memory for their own pool, and latency-sensitive
 * loops where cudaMalloc/cudaFree would synchronise the device. The caller owns every input and
 * output buffer; the engine's scratch is one fixed 32 MiB device array inside the library, held by
 * every GPU that loads it until the process exits. Systems needing more scratch than that
 * (npad * 9 B + 3/8 B per box site + about 140 KB of tables and sub-step entries) are rejected
 * with BFM_ERR_INVALID_ARGUMENT. Boxes are periodic along all three axes. The first
 * call on a device performs a one-time set-up (the scratch's device address) and should come
 * before any stream capture. All calls share the scratch: calls that overlap on the GPU race. */
typedef struct bfm_noalloc_system {
    int32_t* x;                   /* device, npad, in/out: colour-sorted corner positions;  */
    int32_t* y;                   /*   padding slots have x = INT32_MIN                      */
    int32_t* z;
    const uint32_t* nbr;          /* device, maxc * npad: neighbour k of slot g at k*npad + g */
    const uint8_t* nnb;           /* device, npad: neighbour count of each slot */
    uint32_t npad;                /* slots, padding included */
    uint32_t maxc;                /* neighbour slots per monomer, 1..16 */
    uint32_t box[3];              /* powers of two, 4..1024 */
    uint32_t n_colors;            /* colour groups (bfm_color_graph) */
    const uint32_t* group_offset; /* host, n_colors: first slot of each colour group */
    const uint32_t* group_size;   /* host, n_colors: monomers of each group (in-colour index order) */
    const uint8_t* forbidden;     /* host, 512: bond table, 1 = forbidden */
} bfm_noalloc_system;
/* n_mcs MCS of the counter draw stream (seed) starting at sub-step substep0, on `stream` (a
 * cudaStream_t, may be NULL), with the same kernels and results as bfm_run. Calls no
 * cudaMalloc/cudaFree and allocates no host memory; returns once the work is queued. On error,
 * a message goes to err (err_len bytes) if err is not NULL. */
int bfm_sweep_noalloc(const bfm_noalloc_system* s, int32_t n_mcs, uint64_t seed, uint64_t substep0, void* stream,
                      char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* BFM_H */
