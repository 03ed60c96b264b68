// Host side of the BFM sweep engine: the updater behind the reference's API
// (src/pscbfm/UpdaterGPUScBFM_AB_Type.h:316-358), a batch of updaters advanced together, and the
// pieces they share. Everything here is plain C++ over the CUDA runtime; the C-ABI in
// bfm_capi.cpp is a thin exception-to-status layer on top.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfm_device.cuh"
#include "bfm_kernels.hpp"

namespace bfm {

// Error classes, mapped to status codes by the C-ABI. The reference throws std::invalid_argument
// and std::runtime_error for misuse and calls exit() on CUDA errors
// (src/pscbfm/cudacommon.hpp:31-46); here CUDA errors become CudaError.
struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, char const* what);

std::vector<uint8_t> colour_bond_graph(uint32_t n, uint32_t const* cnt, uint32_t const* ids, uint32_t stride);

// Offsets of a system's device arrays in its arena (each array on a 256-byte boundary) and the
// arena's size. Updater::initialize lays its arena out with it; Server::estimateBytes bounds a
// job's device bytes with it before the job is coloured.
struct ArenaLayout {
    size_t x, y, z, nbr, nnb, flags, mark, lat, tmp, tab, grp, stats, desc, steps, list, gs;
    size_t rec, nbrr, plane, moveOk, dir, mlist, mword, mcount, slotOf, xyzOut, snap;
    uint32_t segs;   // mover-list segments (tiles) per parity
    size_t bytes;
};
ArenaLayout arena_layout(uint32_t n, uint32_t npad, uint32_t maxc, uint32_t nwords, uint32_t ntab,
                         uint32_t nColors, uint32_t maxGroup, uint32_t codeMode);
// Bytes of the observables arena of a system (Updater::buildObservables).
size_t observables_bytes(uint32_t npad, uint32_t nMol);

// Host draw stream: per sub-step one draw for the colour (draw % nColors) and one for the seed,
// in that order (src/pscbfm/CRITICAL.cu:509-510).
enum DrawKind : int { kDrawCounter = 0, kDrawCallback = 1 };
using DrawFn = uint32_t (*)(void*);

// The counter stream's draws: counter_draw (bfm_device.cuh).

// Engine path of one updater's run().
enum Mode : int {
    kModeAuto = 0,      // by size: resident, cluster, persistent or graph (autoMode)
    kModeLaunch = 1,    // two kernel launches per sub-step, like the reference
    kModeGraph = 2,     // the same kernels captured into a CUDA graph per chunk of sub-steps
    kModeResident = 3,  // one CTA runs the whole chunk, lattice in shared memory
    kModePersistent = 4,   // bond codes: one cooperative launch per chunk, grid barriers between phases
    kModeCluster = 5,      // bond codes: one cluster of CTAs holds the system in shared memory
};

class Updater {
public:
    explicit Updater(int gpu);
    ~Updater();
    Updater(Updater const&) = delete;
    Updater& operator=(Updater const&) = delete;

    // ---- reference setter API (UpdaterGPUScBFM_AB_Type.h:340-358)
    void setGpu(int gpu);
    void setPeriodicity(bool px, bool py, bool pz);
    void setNrOfAllMonomers(uint32_t n);
    void setAttribute(uint32_t i, int32_t a);
    void setMonomerCoordinates(uint32_t i, int32_t x, int32_t y, int32_t z);
    void setConnectivity(uint32_t a, uint32_t b);
    void setLatticeSize(uint32_t bx, uint32_t by, uint32_t bz);
    void copyBondSet(int dx, int dy, int dz, bool forbidden);
    void populateLattice();
    void initialize();
    void runSimulationOnGPU(int32_t nMcs);   // enqueue + wait, like the reference
    int32_t getMonomerPosition(uint32_t i, int axis);
    void cleanup();

    // ---- engine extensions
    void checkSetup() const;                 // the checks initialize() makes before touching the GPU
    void copySetup(Updater const& other);    // setter state of another (uninitialised) updater
    uint32_t maxNeighbours() const;
    uint64_t boxVolume() const { return (uint64_t)box_[0] * box_[1] * box_[2]; }
    uint32_t boxSide(int a) const { return box_[a]; }
    // side of the occupancy lattice along axis a: the box side, or for a walled axis whose side is
    // not a power of two the next power of two (the box sits in its lowest cells)
    uint32_t latticeSide(int a) const;
    uint64_t latticeVolume() const { return (uint64_t)latticeSide(0) * latticeSide(1) * latticeSide(2); }
    // molecules (connected components of the bond graph) of the current set-up, on the host
    uint32_t countMolecules() const;
    void setCoordinates(int32_t const* xyz, uint32_t n);
    void getCoordinates(int32_t* xyz, uint32_t n);
    void setDrawCounter(uint64_t seed);
    void setDrawCallback(DrawFn fn, void* ctx);
    void setMode(int mode);
    // CTA size of the bond-code check on the grid paths (128, 256, 512; 0: the default 256)
    void setGridBlock(int block);
    int gridBlock() const { return gridBlock_; }
    // the bond-code perform's warps per CTA and per tile (perform_shape_ok; 0, 0: the default)
    void setPerformShape(int warps, int group);
    // a system that only a Batch advances skips the pinned staging of its own run paths
    // (allocated on first use if it runs alone after all)
    void setBatchOnly(bool on) { batchOnly_ = on; }
    int mode() const { return mode_; }
    void run(int32_t nMcs);                  // enqueue only
    void synchronize();
    uint32_t nColors() const;
    std::vector<uint32_t> groupSizes() const;
    void stats(uint64_t out[4]);             // attempted, tentative, accepted, MCS done
    // the counters read without waiting for later work: statsEnqueue queues their copy after the
    // work queued so far and returns a ticket, statsWait waits for that copy only (the last
    // kStatRing tickets stay valid)
    static constexpr uint32_t kStatRing = 8;
    uint64_t statsEnqueue();
    void statsWait(uint64_t ticket, uint64_t out[4]);
    uint64_t substep() const { return subStep_; }
    uint64_t mcsDone() const { return mcsDone_; }
    uint64_t subStep() const { return subStep_; }
    void setSubStep(uint64_t t);   // position of the counter draw stream (after initialize)
    cudaStream_t stream() const { return stream_; }
    bool initialized() const { return dev_.arena != nullptr; }
    uint32_t nMonomers() const { return n_; }
    size_t deviceBytes() const { return dev_.bytes; }
    uint32_t maxGroup() const { return maxGroup_; }
    bool residentEligible() const;
    bool clusterEligible() const { return clusterLogC_ != 0; }
    // the cluster-resident kernel's plan: log2 CTAs per cluster, chunks per warp, shared memory,
    // and whether BFM_MODE_AUTO (clusterFast) or a Batch (clusterForBatch) takes it (planCluster)
    uint32_t clusterLogC() const { return clusterLogC_; }
    uint32_t clusterPer() const { return clusterPer_; }
    size_t clusterSmem() const { return clusterSmem_; }
    bool clusterFast() const { return clusterTier_ >= 3; }
    bool clusterForBatch() const { return clusterTier_ >= 2; }
    int gpu() const { return gpu_; }
    void validate();                         // host-side EV and bond-set check (checkSystem)

    // pieces used by Batch
    SysDev const& desc() const { return dev_.h; }
    SysDev* deviceDesc() const { return dev_.dDesc; }
    uint32_t const* sortedSlot() const { return oldToNew_.data(); }
    StepEntry nextStep();                    // consumes the draws of one sub-step
    void scrubPending(cudaStream_t s);       // clears the temporary marks of the last sub-step
    void noteExternalRun(uint64_t subSteps, uint64_t mcs, bool pendingMarks, uint32_t lastColor);
    uint32_t lastColor() const { return lastColor_; }
    void streamWait(cudaEvent_t e);          // orders this system's later work after e
    void flushTickets();                     // tickets waiting for a snapshot: from the counters, now

    // observables (bfm_observables.cu layout; molecules = connected components of the bonds)
    uint32_t nMolecules() const { return nMol_; }
    std::vector<uint32_t> moleculeSizes() const;
    void observables(long long* out);         // computes now, copies obs_words(nMol) int64
    void enqueueObservables(long long* dOut, cudaStream_t s);   // device buffer, no sync
    void observablesAsync(long long* hostPinned);   // computes and copies on this system's stream, no sync
    void resetReference();                    // MSD reference := current positions

    // measurement
    float runTimed(int32_t nMcs);            // run + CUDA-event time on the handle's stream (ms)
    // the next persistent launch starts its barrier count where no barrier completes (tests)
    void injectBarrierStall() { stallNext_ = true; }
    int path() const;                        // the path the next run takes (BFM_MODE_*)
    void timeKernels(int32_t nMcs, double out[4]);   // check ms, perform ms, launches of each
    uint64_t launches() const { return launches_; }  // kernels launched by this handle so far
    // bytes the run and read-back calls have moved host -> device and device -> host so far
    // (step entries, chain starts, positions, move counters; not the set-up's uploads)
    uint64_t h2dBytes() const { return h2dBytes_; }
    uint64_t d2hBytes() const { return d2hBytes_; }
    void addLaunches(uint64_t n) { launches_ += n; }

private:
    struct Device {
        void* arena = nullptr;
        size_t bytes = 0;
        SysDev h{};
        SysDev* dDesc = nullptr;
        StepEntry* dSteps = nullptr;
        uint32_t stepCap = 0;
        uint32_t* dList = nullptr;     // resident kernel system list (one entry: 0)
        GridSync* gs = nullptr;        // grid barrier of the persistent kernel
        uint32_t* slotOf = nullptr;    // [n] sorted slot of each monomer (caller's order)
        int32_t* xyzOut = nullptr;     // [3 n] positions in the caller's order, for read-back
        unsigned long long* snap = nullptr;      // [kSnapRing][4] counter snapshots of graph replays
        unsigned long long* snapSeq = nullptr;   // snapshots taken so far
    };
    void requireN(char const* who) const;
    void requireInit(char const* who) const;
    void pullPositions();
    void downloadPositions(int32_t* out);   // positions in the caller's order, x y z interleaved
    void enqueueLaunch(uint32_t nSteps);
    void enqueueGraph(uint32_t nSteps);
    void enqueueResident(uint32_t nSteps);
    void enqueueCluster(uint32_t nSteps);
    void planCluster();   // the cluster size and chunks per warp of the cluster-resident kernel
    void enqueuePersistent(uint32_t nSteps);
    void fillSteps(uint32_t nSteps, StepEntry* hostBuf, bool residentParity);
    void freeDevice();
    void ensureStaging();

    int gpu_ = 0;
    cudaStream_t stream_ = nullptr;
    uint32_t n_ = 0;
    bool nSet_ = false;
    std::vector<int32_t> xyz_;                 // host copy, original order
    std::vector<int32_t> attr_;
    std::vector<uint32_t> nbrCnt_;
    std::vector<uint32_t> nbrIds_;             // [n][kMaxConn]
    uint32_t box_[3] = {0, 0, 0};
    uint32_t walls_ = 0;   // bit a: axis a is not periodic
    bool forbidden_[512];
    bool latticePopulated_ = false;

    int drawKind_ = kDrawCounter;
    uint64_t drawSeed_ = 0;
    DrawFn drawFn_ = nullptr;
    void* drawCtx_ = nullptr;
    int mode_ = kModeAuto;
    bool batchOnly_ = false;

    // after initialize
    std::vector<uint8_t> colour_;
    std::vector<uint32_t> grpOff_, grpSize_;
    std::vector<uint32_t> oldToNew_;
    uint32_t npad_ = 0, maxc_ = 1, maxGroup_ = 0;
    uint64_t subStep_ = 0, mcsDone_ = 0;
    uint32_t lastColor_ = kNoColor;            // colour whose marks are still in tmp[(subStep-1)&1]
    bool hostStale_ = false;
    Device dev_;
    StepEntry* hSteps_ = nullptr;              // pinned staging for step entries
    StepGen* hGen_ = nullptr;                  // pinned staging of a chain's start: producer + first entry
    cudaEvent_t genFree_ = nullptr;            // hGen_ may be rewritten after this event
    // the device's entry chain (graph path, counter stream): slot 0 holds the entry of sub-step
    // chainSub_ with previous colour chainPrev_ of the stream of chainSeed_ while chainValid_
    bool chainValid_ = false;
    uint64_t chainSub_ = 0, chainSeed_ = 0;
    uint32_t chainPrev_ = kNoColor;
    uint32_t genOn_ = 0;                       // the device producer's `on`, as last written
    GridSync* hGs_ = nullptr;                  // pinned copy of the persistent kernel's barrier state
    unsigned long long* hStats_ = nullptr;     // pinned copy of the move counters (stats)
    unsigned long long* hStatRing_ = nullptr;  // kStatRing mapped pinned slots (statsEnqueue)
    unsigned long long* dStatRing_ = nullptr;  // the same, as the device addresses them
    unsigned long long* dStats_ = nullptr;     // hStats_ as the device addresses it
    cudaEvent_t statEv_[kStatRing] = {};
    uint64_t statTicket_[kStatRing] = {}, statMcs_[kStatRing] = {}, statNext_ = 0;
    // Once a ticket has been taken (snapMode_), every graph replay takes a snapshot of the counters:
    // with bond codes its first check does, of the counters as the work before the replay left
    // them, so a ticket taken right after a replay waits (pendingTickets_) for the next replay and
    // is then copied from that replay's snapshot into host memory on pubStream_, off the sweep's
    // stream; any other work that changes the counters first publishes the waiting tickets from the
    // counters themselves on the sweep's stream (flushTickets), as does a wait for such a ticket.
    // On the gather representation the replay ends with a snapshot node (k_snapshot_stats) and a
    // ticket taken right after it copies that snapshot at once.
    uint64_t statSeq_[kStatRing] = {};   // expected snapshot sequence of a ticket (0: direct read)
    uint64_t snapIssued_ = 0;            // snapshots enqueued (= the device's snapshot count)
    bool lastRunSnap_ = false;           // the last work changing the counters ended with a snapshot
    bool lastRunLead_ = false;           // ... was a replay whose successor's check takes the snapshot
    bool snapMode_ = false;              // the graphs take counter snapshots
    std::vector<uint32_t> pendingTickets_;   // ticket ring slots waiting for the next snapshot
    void publishPending(uint64_t snapSeq);   // the waiting tickets from snapshot snapSeq, on pubStream_
    bool leadSnapshots() const { return codeMode_ != kCodeNone; }
    cudaStream_t pubStream_ = nullptr;
    cudaEvent_t pubEv_ = nullptr;
    bool gsPending_ = false;                   // hGs_ is being refreshed by the stream
    bool stallNext_ = false;                   // injectBarrierStall
    uint32_t smCount_ = 148;                   // SMs of the device (setGpu)
    uint32_t clusterLogC_ = 0;                 // cluster of 2^logC CTAs holds the system (0: does not fit)
    uint32_t clusterPer_ = 0;                  // chunks of 32 slots per warp and colour
    size_t clusterSmem_ = 0;                   // dynamic shared memory per CTA
    uint32_t clusterTier_ = 0;                 // 3: AUTO takes the plan, 2: a Batch does, 1: forced only
    uint32_t hStepCap_ = 0;
    struct GraphExec {
        uint32_t nSteps, parity0;               // chunk length, parity of its first sub-step
        bool snap;                              // ends with a counter snapshot
        cudaGraphExec_t exec;
    };
    std::vector<GraphExec> graphs_;
    cudaEvent_t stepsFree_ = nullptr;          // host staging may be rewritten after this event
    uint64_t launches_ = 0;
    uint64_t h2dBytes_ = 0, d2hBytes_ = 0;
    int gridBlock_ = 0;
    int perfWarps_ = 0, perfGroup_ = 0;
    void dropGraphs();
    int repr_ = 0;
    uint32_t codeMode_ = kCodeNone;
    uint32_t nMol_ = 0;
    std::vector<uint32_t> molSize_;
    void* obsArena_ = nullptr;
    ObsDev obs_{};
    long long* dObsOut_ = nullptr;
    void buildObservables();
    std::vector<uint32_t> moleculeRoots() const;   // lowest monomer id of each monomer's molecule
    cudaGraphExec_t graphFor(uint32_t nSteps, uint32_t parity0, bool snap);
    void seedChain(cudaStream_t s);           // the device chain restarts at the host's position
    void producerOff(cudaStream_t s);         // the device producer stops writing entries
    int effectiveMode() const;                // the path run() takes (mode_ with AUTO resolved)
    int autoMode() const;                     // the path BFM_MODE_AUTO takes for this system
    void prepareGraphs(uint32_t nSteps);      // capture the graphs a graph-path run of nSteps replays
    // bond codes: unfolded positions (slot order) to image offsets in place (SysDev x, y, z)
    void toImageOffsets(std::vector<int32_t>& hx, std::vector<int32_t>& hy, std::vector<int32_t>& hz) const;
    void hostCodes(std::vector<uint32_t>& pk, std::vector<uint8_t>& code, std::vector<uint32_t>& nbrr) const;
    // bond codes: the device records (SlotRec, rec_words 32-bit words each) of host lattice
    // addresses and code words
    std::vector<uint32_t> slotRecords(std::vector<uint32_t> const& pk, std::vector<uint8_t> const& code) const;

public:
    // representation of the bonds on the device: auto (bond codes when the neighbour lists are
    // symmetric and <= 6 per monomer, else neighbour positions) or forced neighbour positions
    static constexpr int kReprAuto = 0, kReprGather = 1;
    void setRepresentation(int r);
    uint32_t codeMode() const { return codeMode_; }
    uint32_t gridTiles() const;                               // CTAs of one grid-phase launch
    cudaError_t launchCheck(StepEntry const* e, cudaStream_t s, unsigned long long* snap = nullptr) const;
    cudaError_t launchPerform(StepEntry const* e, cudaStream_t s, PerformArgs pa) const;
    static PerformArgs performArgs(StepEntry const& e);   // parity and scope of a host-made entry
    size_t residentSmem() const;
};

// A set of initialised updaters on one GPU advanced together: systems that fit one CTA run in the
// resident kernel and systems that fit a cluster of CTAs in the cluster-resident kernel (one
// launch per run and group), the others share one grid-phase launch per phase and sub-step,
// captured into a CUDA graph. Every system keeps its own draw stream, so its
// trajectory is identical to running it alone.
class Batch {
public:
    Batch(int gpu, Updater* const* members, uint32_t n);
    ~Batch();
    void run(int32_t nMcs);     // enqueue
    void run(int32_t const* mcs);   // enqueue mcs[i] MCS of member i (0: the member idles)
    // replaces the member list; streams, events and buffers are kept (buffers grow as needed)
    void setMembers(Updater* const* members, uint32_t n);
    // register budget of the grid-phase kernels (launch_check_bc), -1: the default
    void setShape(int shape);
    int shape() const { return shape_; }
    // CTA size of the grid groups' check (128, 256, 512; 0: the default)
    void setBlock(int block);
    int block() const { return block_; }
    // the grid groups' perform: warps per CTA and per tile (perform_shape_ok; 0, 0: the default)
    void setPerformShape(int warps, int group);
    int performWarps() const { return perfWarps_; }
    int performGroup() const { return perfGroup_; }
    bool residentEnabled() const { return residentOn_; }
    bool clusterEnabled() const { return clusterOn_; }
    // Runs the members under each configuration (kernel shape x resident path on / off x cluster
    // path on / off) for 1 + mcsPerTrial MCS, keeps the fastest per MCS and returns every trial.
    // The MCS count as ordinary steps of the run: the results do not depend on the configuration.
    struct Trial {
        int shape;
        bool resident;
        bool cluster;
        int block;
        int perfWarps, perfGroup;
        float msPerMcs;
    };
    std::vector<Trial> autotune(int32_t mcsPerTrial);
    float runTimed(int32_t nMcs);   // run + CUDA-event time on the batch stream (ms)
    void synchronize();
    uint32_t size() const { return (uint32_t)members_.size(); }
    Updater* member(uint32_t i) const { return members_.at(i); }
    void setResidentEnabled(bool on)
    {
        if (on != residentOn_) built_ = false;
        residentOn_ = on;
    }
    // members too large for one CTA whose cluster plan beats the grid-phase kernels
    // (Updater::clusterForBatch: at most two chunks of 32 slots per warp and colour) run in the
    // cluster-resident kernel, while the batch's clusters take at most half of the SMs (the rest
    // stay with the grid-phase kernels)
    void setClusterEnabled(bool on)
    {
        if (on != clusterOn_) built_ = false;
        clusterOn_ = on;
    }
    cudaStream_t stream() const { return stream_; }
    uint32_t residentCount() const;
    uint32_t clusterCount() const;
    uint64_t launches() const { return launches_; }

private:
    // members of one representation (codeMode) on one path
    struct GridGroup {
        uint32_t codeMode;
        std::vector<TileRef> tiles;
        TileRef* dTiles = nullptr;
        std::vector<TileRef> ptiles;     // the perform's list (bond codes: tiles grouped, perform_tile_list)
        TileRef* dPTiles = nullptr;
        std::vector<uint32_t> members;   // batch indices of the group's systems
    };
    struct ResidentGroup {
        uint32_t codeMode;
        std::vector<uint32_t> members;
        uint32_t* dList = nullptr;
        uint32_t perThread = 1;
        size_t smem = 0;
    };
    // members of one representation with the same cluster size, one launch per run on a stream
    // of their own (side_[side])
    struct ClusterGroup {
        uint32_t codeMode;
        uint32_t logC;
        std::vector<uint32_t> members;
        uint32_t* dList = nullptr;
        uint32_t perThread = 1;
        size_t smem = 0;
        size_t side = 0;
    };
    void rebuild();
    void validateMembers(Updater* const* members, uint32_t n) const;
    cudaError_t launchGrid(StepEntry const* e);   // one sub-step of every grid group, entries [members]
    void reserveSteps(size_t entries);           // host staging and device entries for a run
    void ensureGraph();                          // capture the graph of stepCap_ sub-steps
    void prepare(int32_t const* mcs);            // both, for a run of mcs[i] MCS per member
    int gpu_;
    std::vector<Updater*> members_;
    std::vector<char> wholeRun_;               // member runs in a resident or cluster kernel
    std::vector<GridGroup> grid_;
    std::vector<ResidentGroup> resident_;
    std::vector<ClusterGroup> cluster_;
    std::vector<cudaStream_t> side_;           // streams of the cluster groups (grown, never shrunk)
    std::vector<cudaEvent_t> sideJoin_;
    uint32_t smCount_ = 148;
    bool residentOn_ = true;
    bool clusterOn_ = true;
    bool built_ = false;
    int shape_ = -1;
    int block_ = 0;
    int perfWarps_ = 0, perfGroup_ = 0;
    cudaStream_t stream_ = nullptr, stream2_ = nullptr;
    cudaEvent_t join_ = nullptr, fork_ = nullptr, ready_ = nullptr;
    void* arena_ = nullptr;                    // descriptors, graph window, tiles, lists
    size_t arenaBytes_ = 0, hStepsCap_ = 0, dStepsCap_ = 0;
    SysDev* dSys_ = nullptr;                   // descriptors of all members
    StepEntry* dWindow_ = nullptr;             // [stepCap_][members]: entries the captured graph reads
    StepEntry* dStepsAll_ = nullptr;           // [sub-steps of the run][members]
    StepEntry* hSteps_ = nullptr;              // pinned staging of dStepsAll_
    size_t stepCap_ = 0;
    cudaEvent_t stepsFree_ = nullptr;
    cudaEvent_t done_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    uint64_t launches_ = 0;
};

}  // namespace bfm
