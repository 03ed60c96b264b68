// Batch: many independent systems advanced together on one GPU.
//
// Systems whose lattices (and, in the bond-code representation, packed coordinates and bond
// codes) fit one CTA's shared memory run in the resident kernel, one CTA per system, one launch
// per run. Systems of the bond-code representation that a cluster of 2-16 CTAs holds in its
// distributed shared memory with at most two chunks of 32 slots per warp and colour (where that
// kernel beats the grid-phase kernels) run in the cluster-resident kernel, one cluster per system and one
// launch per run and cluster size, while the batch's clusters take at most half of the SMs. The
// other systems share the grid-phase kernels: one check and one perform launch per
// sub-step and representation cover the active colour group of every such system at once, and
// chunks of those launches are captured into a CUDA graph once and replayed. Each system draws its
// own sub-steps from its own stream exactly as it would alone, so its trajectory is unchanged by
// batching.
//
// A run stages the step entries of all its sub-steps with one host-to-device copy; the resident
// and the grid-phase launches then proceed on two streams without meeting until the run ends, and
// the host returns as soon as the work is queued. Each cluster group runs on a stream of its own. Member streams are ordered before the run and
// after it with events, never with host waits.

#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "bfm_engine.hpp"

namespace bfm {

namespace {
constexpr uint32_t kBatchChunk = 64;      // sub-steps per captured graph of the grid phase
size_t up256(size_t v) { return (v + 255) & ~size_t(255); }
}  // namespace

Batch::Batch(int gpu, Updater* const* members, uint32_t n) : gpu_(gpu)
{
    validateMembers(members, n);
    members_.assign(members, members + n);
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking), "cudaStreamCreate");
    for (cudaEvent_t* e : {&join_, &fork_, &stepsFree_, &done_, &ready_})
        cuda_check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu_) == cudaSuccess && sms > 0)
        smCount_ = (uint32_t)sms;
}

Batch::~Batch()
{
    cudaSetDevice(gpu_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (stream2_) cudaStreamSynchronize(stream2_);
    for (cudaStream_t q : side_) cudaStreamSynchronize(q);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (arena_) cudaFreeAsync(arena_, stream_);
    if (dStepsAll_) cudaFreeAsync(dStepsAll_, stream_);
    if (stream_) cudaStreamSynchronize(stream_);
    cudaFreeHost(hSteps_);
    for (cudaEvent_t e : {join_, fork_, stepsFree_, done_, ready_})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : sideJoin_) cudaEventDestroy(e);
    for (cudaStream_t q : side_) cudaStreamDestroy(q);
    if (stream_) cudaStreamDestroy(stream_);
    if (stream2_) cudaStreamDestroy(stream2_);
}

uint32_t Batch::residentCount() const
{
    uint32_t n = 0;
    for (auto const& g : resident_) n += (uint32_t)g.members.size();
    return n;
}

uint32_t Batch::clusterCount() const
{
    uint32_t n = 0;
    for (auto const& g : cluster_) n += (uint32_t)g.members.size();
    return n;
}

void Batch::setMembers(Updater* const* members, uint32_t n)
{
    validateMembers(members, n);
    members_.assign(members, members + n);
    built_ = false;
}

void Batch::validateMembers(Updater* const* members, uint32_t n) const
{
    if (n == 0) throw std::invalid_argument("[Batch] no systems");
    for (uint32_t i = 0; i < n; ++i) {
        Updater* u = members[i];
        if (!u) throw std::invalid_argument("[Batch] null system");
        if (!u->initialized()) throw std::runtime_error("[Batch] every system must be initialized");
        if (u->gpu() != gpu_) throw std::invalid_argument("[Batch] every system must live on the batch GPU");
        for (uint32_t j = 0; j < i; ++j)
            if (members[j] == u) throw std::invalid_argument("[Batch] a system appears twice");
    }
}

void Batch::rebuild()
{
    // the previous launches may still read the arena
    cuda_check(cudaStreamSynchronize(stream_), "batch");
    cuda_check(cudaStreamSynchronize(stream2_), "batch");
    for (cudaStream_t q : side_) cuda_check(cudaStreamSynchronize(q), "batch");
    uint32_t const M = (uint32_t)members_.size();
    grid_.clear();
    resident_.clear();
    cluster_.clear();
    wholeRun_.assign(M, 0);
    auto gridGroup = [&](uint32_t mode) -> GridGroup& {
        for (auto& g : grid_)
            if (g.codeMode == mode) return g;
        grid_.push_back(GridGroup{mode, {}, nullptr, {}, nullptr, {}});
        return grid_.back();
    };
    auto resGroup = [&](uint32_t mode) -> ResidentGroup& {
        for (auto& g : resident_)
            if (g.codeMode == mode) return g;
        resident_.push_back(ResidentGroup{mode, {}, nullptr, 1, 0});
        return resident_.back();
    };
    auto clusterGroup = [&](uint32_t mode, uint32_t logC) -> ClusterGroup& {
        for (auto& g : cluster_)
            if (g.codeMode == mode && g.logC == logC) return g;
        cluster_.push_back(ClusterGroup{mode, logC, {}, nullptr, 1, 0, cluster_.size()});
        return cluster_.back();
    };
    uint32_t clusterCtas = 0;
    for (uint32_t m = 0; m < M; ++m) {
        Updater* u = members_[m];
        uint32_t const C = 1u << u->clusterLogC();
        if (residentOn_ && u->residentEligible()) {
            ResidentGroup& g = resGroup(u->codeMode());
            g.members.push_back(m);
            g.smem = std::max(g.smem, u->residentSmem());
            while (g.perThread * kResidentBlock < u->maxGroup()) g.perThread *= 2;
            wholeRun_[m] = 1;
        } else if (clusterOn_ && u->clusterEligible() && u->clusterForBatch() && clusterCtas + C <= smCount_ / 2u) {
            ClusterGroup& g = clusterGroup(u->codeMode(), u->clusterLogC());
            g.members.push_back(m);
            g.smem = std::max(g.smem, u->clusterSmem());
            g.perThread = std::max(g.perThread, u->clusterPer());
            clusterCtas += C;
            wholeRun_[m] = 1;
        } else {
            GridGroup& g = gridGroup(u->codeMode());
            uint32_t const span = u->codeMode() == kCodeNone ? kGridBlock : kBcTileSpan;
            uint32_t const t = u->gridTiles();
            for (uint32_t k = 0; k < t; ++k) g.tiles.push_back(TileRef{m, k * span});
            g.members.push_back(m);
        }
    }
    for (auto& g : grid_) g.ptiles = g.codeMode == kCodeNone ? g.tiles : perform_tile_list(g.tiles);
    stepCap_ = kBatchChunk;
    size_t total = up256(sizeof(SysDev) * M) + up256(sizeof(StepEntry) * stepCap_ * M);
    for (auto const& g : grid_) total += up256(sizeof(TileRef) * g.tiles.size()) + up256(sizeof(TileRef) * g.ptiles.size());
    for (auto const& g : resident_) total += up256(sizeof(uint32_t) * g.members.size());
    for (auto const& g : cluster_) total += up256(sizeof(uint32_t) * g.members.size());
    while (side_.size() < cluster_.size()) {
        cudaStream_t q = nullptr;
        cudaEvent_t e = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "cudaStreamCreate");
        side_.push_back(q);
        cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        sideJoin_.push_back(e);
    }
    for (auto& g : cluster_) {
        // one launch runs every cluster of the group at one size; a member planned with fewer
        // chunks per warp runs as well with more (the kernel walks only its own chunks)
        size_t smem = 0;
        for (uint32_t m : g.members) {
            Updater const* u = members_[m];
            smem = std::max(smem, cluster_bc_smem_bytes(u->desc().nwords, u->desc().npad, g.logC, g.perThread,
                                                        g.codeMode));
        }
        g.smem = smem;
        if (!cluster_bc_runnable(g.logC, g.perThread, g.smem, g.codeMode))
            throw std::runtime_error("[Batch] a cluster group's configuration does not run on this device");
    }
    if (total > arenaBytes_) {   // grows only: membership changes reuse the arena
        if (arena_) cuda_check(cudaFreeAsync(arena_, stream_), "cudaFreeAsync(batch)");
        arena_ = nullptr;
        arenaBytes_ = 0;
        cuda_check(cudaMallocAsync(&arena_, total * 2, stream_), "cudaMallocAsync(batch)");
        arenaBytes_ = total * 2;
    }
    char* p = static_cast<char*>(arena_);
    dSys_ = reinterpret_cast<SysDev*>(p);
    p += up256(sizeof(SysDev) * M);
    dWindow_ = reinterpret_cast<StepEntry*>(p);
    p += up256(sizeof(StepEntry) * stepCap_ * M);
    std::vector<SysDev> descs(M);
    for (uint32_t m = 0; m < M; ++m) descs[m] = members_[m]->desc();
    cuda_check(cudaMemcpyAsync(dSys_, descs.data(), sizeof(SysDev) * M, cudaMemcpyHostToDevice, stream_),
               "upload descriptors");
    for (auto& g : grid_) {
        g.dTiles = reinterpret_cast<TileRef*>(p);
        p += up256(sizeof(TileRef) * g.tiles.size());
        cuda_check(cudaMemcpyAsync(g.dTiles, g.tiles.data(), sizeof(TileRef) * g.tiles.size(), cudaMemcpyHostToDevice,
                                   stream_),
                   "upload tiles");
        g.dPTiles = reinterpret_cast<TileRef*>(p);
        p += up256(sizeof(TileRef) * g.ptiles.size());
        cuda_check(cudaMemcpyAsync(g.dPTiles, g.ptiles.data(), sizeof(TileRef) * g.ptiles.size(),
                                   cudaMemcpyHostToDevice, stream_),
                   "upload perform tiles");
    }
    for (auto& g : resident_) {
        g.dList = reinterpret_cast<uint32_t*>(p);
        p += up256(sizeof(uint32_t) * g.members.size());
        cuda_check(cudaMemcpyAsync(g.dList, g.members.data(), sizeof(uint32_t) * g.members.size(),
                                   cudaMemcpyHostToDevice, stream_),
                   "upload resident list");
    }
    for (auto& g : cluster_) {
        g.dList = reinterpret_cast<uint32_t*>(p);
        p += up256(sizeof(uint32_t) * g.members.size());
        cuda_check(cudaMemcpyAsync(g.dList, g.members.data(), sizeof(uint32_t) * g.members.size(),
                                   cudaMemcpyHostToDevice, stream_),
                   "upload cluster list");
    }
    // the host vectors above die with this call: finish their copies now
    cuda_check(cudaStreamSynchronize(stream_), "batch uploads");
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    built_ = true;
}

cudaError_t Batch::launchGrid(StepEntry const* e)
{
    SysDev const unused{};   // multi-system launches read each CTA's descriptor from dSys_
    PerformArgs pa;
    pa.warps = perfWarps_;
    pa.group = perfGroup_;
    for (auto const& g : grid_) {
        uint32_t const n = (uint32_t)g.tiles.size();
        if (g.members.size() == 1) {
            // a lone system runs the single-system kernels, as it would alone (descriptor as a launch
            // parameter, several tiles per perform CTA): a long job left alone in a server lane
            // then runs at its own speed
            uint32_t const m = g.members[0];
            Updater const& u = *members_[m];
            cudaError_t err = g.codeMode == kCodeNone
                                  ? launch_check(u.deviceDesc(), nullptr, n, kGridBlock, e + m, stream_)
                                  : launch_check_bc(u.desc(), u.deviceDesc(), nullptr, n, e + m, g.codeMode, stream_, shape_, block_);
            if (err != cudaSuccess) return err;
            err = g.codeMode == kCodeNone
                      ? launch_perform(u.deviceDesc(), nullptr, n, kGridBlock, e + m, stream_)
                      : launch_perform_bc(u.desc(), u.deviceDesc(), nullptr, n, e + m, g.codeMode, stream_, shape_, pa);
            if (err != cudaSuccess) return err;
            continue;
        }
        cudaError_t err = g.codeMode == kCodeNone
                              ? launch_check(dSys_, g.dTiles, n, kGridBlock, e, stream_)
                              : launch_check_bc(unused, dSys_, g.dTiles, n, e, g.codeMode, stream_, shape_, block_);
        if (err != cudaSuccess) return err;
        err = g.codeMode == kCodeNone
                  ? launch_perform(dSys_, g.dTiles, n, kGridBlock, e, stream_)
                  : launch_perform_bc(unused, dSys_, g.dPTiles, (uint32_t)g.ptiles.size(), e, g.codeMode, stream_, shape_, pa);
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

void Batch::reserveSteps(size_t entries)
{
    // the previous run's copy has read the host staging once stepsFree_ has passed
    cuda_check(cudaEventSynchronize(stepsFree_), "batch staging");
    if (entries > hStepsCap_) {
        cudaFreeHost(hSteps_);
        hSteps_ = nullptr;
        hStepsCap_ = 0;
        cuda_check(cudaMallocHost(&hSteps_, sizeof(StepEntry) * entries * 2), "cudaMallocHost(batch steps)");
        hStepsCap_ = entries * 2;
    }
    if (entries > dStepsCap_) {
        if (dStepsAll_) cuda_check(cudaFreeAsync(dStepsAll_, stream_), "cudaFreeAsync(batch steps)");
        dStepsAll_ = nullptr;
        dStepsCap_ = 0;
        cuda_check(cudaMallocAsync(&dStepsAll_, sizeof(StepEntry) * entries * 2, stream_),
                   "cudaMallocAsync(batch steps)");
        dStepsCap_ = entries * 2;
    }
}

void Batch::ensureGraph()
{
    if (graph_) return;
    uint32_t const M = (uint32_t)members_.size();
    cudaGraph_t g;
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaSuccess;
    for (uint32_t t = 0; t < stepCap_ && err == cudaSuccess; ++t) err = launchGrid(dWindow_ + (size_t)t * M);
    cudaError_t const endErr = cudaStreamEndCapture(stream_, &g);
    cuda_check(err, "capture batch launches");
    cuda_check(endErr, "end capture");
    cudaError_t const ie = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    cuda_check(ie, "graph instantiate");
}

void Batch::prepare(int32_t const* mcs)
{
    // one-time host work of a run (staging growth, graph capture), done ahead of a timed run
    uint32_t const M = (uint32_t)members_.size();
    uint64_t T = 0;
    for (uint32_t m = 0; m < M; ++m) T = std::max(T, (uint64_t)std::max(mcs[m], 0) * members_[m]->nColors());
    if (T == 0) return;
    reserveSteps((size_t)T * M);
    if (!grid_.empty() && T >= stepCap_) ensureGraph();
}

void Batch::run(int32_t nMcs)
{
    if (nMcs <= 0) return;
    std::vector<int32_t> each(members_.size(), nMcs);
    run(each.data());
}

void Batch::run(int32_t const* mcs)
{
    uint32_t const M = (uint32_t)members_.size();
    for (uint32_t m = 0; m < M; ++m)
        if (mcs[m] < 0) throw std::invalid_argument("[Batch::run] negative MCS count");
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    if (!built_) rebuild();
    // pending grid-path marks of members that run in a resident or cluster kernel are cleared on
    // their own streams; then the batch waits for every member stream (uploads, scrubs,
    // observables) on the device
    for (uint32_t m = 0; m < M; ++m)
        if (wholeRun_[m]) members_[m]->scrubPending(members_[m]->stream());
    for (Updater* u : members_) {
        u->flushTickets();   // a member's ticket still waiting for a snapshot reads its counters now
        cuda_check(cudaEventRecord(ready_, u->stream()), "event");
        cuda_check(cudaStreamWaitEvent(stream_, ready_, 0), "wait");
    }

    std::vector<uint64_t> need(M);
    uint64_t T = 0;
    for (uint32_t m = 0; m < M; ++m) {
        need[m] = (uint64_t)mcs[m] * members_[m]->nColors();
        T = std::max(T, need[m]);
    }
    if (T > 0) {
        size_t const entries = (size_t)T * M;
        reserveSteps(entries);
        for (uint64_t t = 0; t < T; ++t)
            for (uint32_t m = 0; m < M; ++m) {
                StepEntry& e = hSteps_[(size_t)t * M + m];
                if (t < need[m]) e = members_[m]->nextStep();
                else e = StepEntry{kNoColor, 0u, 0u, kNoColor, 0u, 0u, 0u, 0u};
            }
        cuda_check(cudaMemcpyAsync(dStepsAll_, hSteps_, sizeof(StepEntry) * entries, cudaMemcpyHostToDevice, stream_),
                   "batch steps H2D");
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        if (!resident_.empty() || !cluster_.empty()) cuda_check(cudaEventRecord(fork_, stream_), "event");
        for (auto const& g : cluster_) {
            // one launch per cluster size for the whole run, each on a stream of its own
            cudaStream_t const q = side_[g.side];
            cuda_check(cudaStreamWaitEvent(q, fork_, 0), "wait");
            cuda_check(launch_cluster_bc(dSys_, g.dList, (uint32_t)g.members.size(), g.logC, g.perThread, dStepsAll_,
                                         M, (uint32_t)T, g.smem, g.codeMode, q),
                       "batch cluster");
            cuda_check(cudaEventRecord(sideJoin_[g.side], q), "event");
            ++launches_;
        }
        if (!resident_.empty()) {
            // one launch per group for the whole run, on the second stream
            cuda_check(cudaStreamWaitEvent(stream2_, fork_, 0), "wait");
            for (auto const& g : resident_) {
                cuda_check(g.codeMode == kCodeNone
                               ? launch_resident(dSys_, g.dList, (uint32_t)g.members.size(), g.perThread, dStepsAll_,
                                                 M, (uint32_t)T, g.smem, stream2_)
                               : launch_resident_bc(dSys_, g.dList, (uint32_t)g.members.size(), g.perThread,
                                                    dStepsAll_, M, (uint32_t)T, g.smem, g.codeMode, stream2_),
                           "batch resident");
                ++launches_;
            }
        }
        if (!grid_.empty()) {
            for (uint64_t t0 = 0; t0 < T; t0 += stepCap_) {
                uint32_t const chunk = (uint32_t)std::min<uint64_t>(stepCap_, T - t0);
                if (chunk == stepCap_) {
                    // the captured graph reads its entries from the window
                    cuda_check(cudaMemcpyAsync(dWindow_, dStepsAll_ + t0 * M, sizeof(StepEntry) * stepCap_ * M,
                                               cudaMemcpyDeviceToDevice, stream_),
                               "batch window");
                    ensureGraph();
                    cuda_check(cudaGraphLaunch(graph_, stream_), "batch graph launch");
                } else {
                    for (uint32_t t = 0; t < chunk; ++t)
                        cuda_check(launchGrid(dStepsAll_ + (t0 + t) * M), "batch grid launch");
                }
                launches_ += 2ull * chunk * grid_.size();
            }
        }
        if (!resident_.empty()) {
            cuda_check(cudaEventRecord(join_, stream2_), "event");
            cuda_check(cudaStreamWaitEvent(stream_, join_, 0), "wait");
        }
        for (auto const& g : cluster_) cuda_check(cudaStreamWaitEvent(stream_, sideJoin_[g.side], 0), "wait");
    }
    cuda_check(cudaEventRecord(done_, stream_), "event");
    for (uint32_t m = 0; m < M; ++m) {
        members_[m]->noteExternalRun(need[m], (uint64_t)mcs[m], !wholeRun_[m], members_[m]->lastColor());
        members_[m]->streamWait(done_);
    }
}

void Batch::setShape(int shape)
{
    if (shape >= kGridShapes) throw std::invalid_argument("[Batch::setShape] unknown kernel shape");
    if (shape != shape_) built_ = false;   // the captured graph holds the old kernels
    shape_ = shape;
}

void Batch::setBlock(int block)
{
    if (block != 0 && !check_block_ok(block))
        throw std::invalid_argument("[Batch::setBlock] the check's CTA size must be 128, 256 or 512 threads");
    if (block != block_) built_ = false;   // the captured graph holds the old kernels
    block_ = block;
}

void Batch::setPerformShape(int warps, int group)
{
    if (!perform_shape_ok(warps, group))
        throw std::invalid_argument("[Batch::setPerformShape] warps per CTA and per tile must be 1, 2, 4 or 8, "
                                    "the second at most the first (0, 0: the default)");
    if (warps != perfWarps_ || group != perfGroup_) built_ = false;   // the captured graph holds the old kernels
    perfWarps_ = warps;
    perfGroup_ = group;
}

std::vector<Batch::Trial> Batch::autotune(int32_t mcsPerTrial)
{
    // Every configuration gives the same trajectories, so the trials are ordinary MCS of the run:
    // each configuration runs 1 MCS (graph capture, warm-up) and then mcsPerTrial timed MCS.
    if (mcsPerTrial <= 0) throw std::invalid_argument("[Batch::autotune] trials need at least one MCS");
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    if (!built_) rebuild();
    // cluster on and off differ only where a member that does not run resident could run in a
    // cluster
    bool anyResident = false, anyCluster[2] = {false, false};
    for (Updater* u : members_) {
        anyResident = anyResident || u->residentEligible();
        bool const cl = u->clusterEligible() && u->clusterForBatch();
        anyCluster[0] = anyCluster[0] || cl;
        anyCluster[1] = anyCluster[1] || (cl && !u->residentEligible());
    }
    // Three stages, each configuration timed over the same kind of MCS: first the paths (resident
    // kernel on / off x cluster kernel on / off, where either can matter) with the grid kernels'
    // defaults; then, for the best paths and if some member runs on the grid-phase kernels, the
    // check's register budget (kGridShapes) x its CTA size (128, 256, 512 threads), as the
    // reference sweeps its block size (CRITICAL.cu:445-487); last, for the best of those, the
    // perform's warps per CTA x warps per tile.
    std::vector<Trial> trials;
    auto time_it = [&](bool resident, bool cl, int shape, int block, int pw, int pg) {
        setResidentEnabled(resident);
        setClusterEnabled(cl);
        setShape(shape);
        setBlock(block);
        setPerformShape(pw, pg);
        rebuild();
        runTimed(1);
        trials.push_back(
            Trial{shape_, resident, cl, block_, pw, pg, runTimed(mcsPerTrial) / (float)mcsPerTrial});
        return trials.back();
    };
    Trial best{};
    bool first = true;
    for (int resident = 1; resident >= 0; --resident) {
        if (!resident && !anyResident) break;   // the same configuration as resident on
        for (int cl = 1; cl >= 0; --cl) {
            if (!cl && !anyCluster[resident]) break;   // the same configuration as cluster on
            Trial const t = time_it(resident != 0, cl != 0, -1, 0, 0, 0);
            if (first || t.msPerMcs < best.msPerMcs) best = t;
            first = false;
        }
    }
    setResidentEnabled(best.resident);
    setClusterEnabled(best.cluster);
    rebuild();
    if (!grid_.empty()) {
        for (int block : {128, 256, 512})
            for (int sh = 0; sh < kGridShapes; ++sh) {
                Trial const t = time_it(best.resident, best.cluster, sh, block, 0, 0);
                if (t.msPerMcs < best.msPerMcs) best = t;
            }
        Trial const base = best;
        for (auto pw : kPerformShapeTrials) {
            Trial const t = time_it(base.resident, base.cluster, base.shape, base.block, pw[0], pw[1]);
            if (t.msPerMcs < best.msPerMcs) best = t;
        }
    }
    setResidentEnabled(best.resident);
    setClusterEnabled(best.cluster);
    setShape(best.shape);
    setBlock(best.block);
    setPerformShape(best.perfWarps, best.perfGroup);
    return trials;
}

float Batch::runTimed(int32_t nMcs)
{
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    for (Updater* u : members_) u->synchronize();
    if (!built_) rebuild();
    if (nMcs > 0) {
        std::vector<int32_t> each(members_.size(), nMcs);
        prepare(each.data());
    }
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "cudaEventCreate");
    cuda_check(cudaEventCreate(&b), "cudaEventCreate");
    cuda_check(cudaEventRecord(a, stream_), "event");
    run(nMcs);   // the resident stream joins stream_ before run() returns
    cuda_check(cudaEventRecord(b, stream_), "event");
    cuda_check(cudaEventSynchronize(b), "timed batch");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, a, b), "elapsed");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

void Batch::synchronize()
{
    cuda_check(cudaStreamSynchronize(stream_), "batch");
    cuda_check(cudaStreamSynchronize(stream2_), "batch");
}

}  // namespace bfm
