// Batch: many independent systems advanced together on one GPU.
//
// Systems whose lattices (and, in the bond-code representation, packed coordinates and bond
// codes) fit one CTA's shared memory run in the resident kernel, one CTA per system, one launch
// per chunk of sub-steps. The other systems share the grid-phase kernels: one check and one
// perform launch per sub-step and representation cover the active colour group of every such
// system at once, and a chunk of those launches is captured into a CUDA graph once and replayed.
// The two paths run concurrently on two streams. Each system draws its own sub-steps from its own
// stream exactly as it would alone, so its trajectory is unchanged by batching.

#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "bfm_engine.hpp"

namespace bfm {

namespace {
constexpr uint32_t kBatchChunk = 64;      // sub-steps per staged chunk / per captured graph
size_t up256(size_t v) { return (v + 255) & ~size_t(255); }
}  // namespace

Batch::Batch(int gpu, Updater* const* members, uint32_t n) : gpu_(gpu)
{
    validateMembers(members, n);
    members_.assign(members, members + n);
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&stepsFree_, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "cudaEventCreate");
}

Batch::~Batch()
{
    cudaSetDevice(gpu_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (stream2_) cudaStreamSynchronize(stream2_);
    if (graph_) cudaGraphExecDestroy(graph_);
    cudaFree(arena_);
    cudaFreeHost(hSteps_);
    for (cudaEvent_t e : {join_, fork_, stepsFree_, done_})
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
    if (stream2_) cudaStreamDestroy(stream2_);
}

uint32_t Batch::residentCount() const
{
    uint32_t n = 0;
    for (auto const& g : resident_) n += (uint32_t)g.members.size();
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
    // the previous launches may still read the arena and the staging buffer
    cuda_check(cudaStreamSynchronize(stream_), "batch");
    cuda_check(cudaStreamSynchronize(stream2_), "batch");
    uint32_t const M = (uint32_t)members_.size();
    grid_.clear();
    resident_.clear();
    isResident_.assign(M, 0);
    auto gridGroup = [&](uint32_t mode) -> GridGroup& {
        for (auto& g : grid_)
            if (g.codeMode == mode) return g;
        grid_.push_back(GridGroup{mode, {}, nullptr});
        return grid_.back();
    };
    auto resGroup = [&](uint32_t mode) -> ResidentGroup& {
        for (auto& g : resident_)
            if (g.codeMode == mode) return g;
        resident_.push_back(ResidentGroup{mode, {}, nullptr, 1, 0});
        return resident_.back();
    };
    for (uint32_t m = 0; m < M; ++m) {
        Updater* u = members_[m];
        if (residentOn_ && u->residentEligible()) {
            ResidentGroup& g = resGroup(u->codeMode());
            g.members.push_back(m);
            g.smem = std::max(g.smem, u->residentSmem());
            while (g.perThread * kResidentBlock < u->maxGroup()) g.perThread *= 2;
            isResident_[m] = 1;
        } else {
            GridGroup& g = gridGroup(u->codeMode());
            uint32_t const span = u->codeMode() == kCodeNone ? kGridBlock : kBcTileSpan;
            uint32_t const t = u->gridTiles();
            for (uint32_t k = 0; k < t; ++k) g.tiles.push_back(TileRef{m, k * span});
        }
    }
    stepCap_ = kBatchChunk;
    size_t total = up256(sizeof(SysDev) * M) + up256(sizeof(StepEntry) * stepCap_ * M);
    for (auto const& g : grid_) total += up256(sizeof(TileRef) * g.tiles.size());
    for (auto const& g : resident_) total += up256(sizeof(uint32_t) * g.members.size());
    if (total > arenaBytes_) {   // grows only: membership changes reuse the arena
        cudaFree(arena_);
        arena_ = nullptr;
        arenaBytes_ = 0;
        cuda_check(cudaMalloc(&arena_, total), "cudaMalloc(batch)");
        arenaBytes_ = total;
    }
    char* p = static_cast<char*>(arena_);
    dSys_ = reinterpret_cast<SysDev*>(p);
    p += up256(sizeof(SysDev) * M);
    dSteps_ = reinterpret_cast<StepEntry*>(p);
    p += up256(sizeof(StepEntry) * stepCap_ * M);
    std::vector<SysDev> descs(M);
    for (uint32_t m = 0; m < M; ++m) descs[m] = members_[m]->desc();
    cuda_check(cudaMemcpy(dSys_, descs.data(), sizeof(SysDev) * M, cudaMemcpyHostToDevice), "upload descriptors");
    for (auto& g : grid_) {
        g.dTiles = reinterpret_cast<TileRef*>(p);
        p += up256(sizeof(TileRef) * g.tiles.size());
        cuda_check(cudaMemcpy(g.dTiles, g.tiles.data(), sizeof(TileRef) * g.tiles.size(), cudaMemcpyHostToDevice),
                   "upload tiles");
    }
    for (auto& g : resident_) {
        g.dList = reinterpret_cast<uint32_t*>(p);
        p += up256(sizeof(uint32_t) * g.members.size());
        cuda_check(cudaMemcpy(g.dList, g.members.data(), sizeof(uint32_t) * g.members.size(), cudaMemcpyHostToDevice),
                   "upload resident list");
    }
    if (stepCap_ * M > hStepsCap_) {
        cuda_check(cudaEventSynchronize(stepsFree_), "batch staging");
        cudaFreeHost(hSteps_);
        hSteps_ = nullptr;
        hStepsCap_ = 0;
        cuda_check(cudaMallocHost(&hSteps_, sizeof(StepEntry) * stepCap_ * M * 2), "cudaMallocHost(batch steps)");
        hStepsCap_ = stepCap_ * M * 2;
    }
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    built_ = true;
}

cudaError_t Batch::launchGrid(uint32_t t, uint32_t M)
{
    StepEntry const* e = dSteps_ + (size_t)t * M;
    SysDev const unused{};   // multi-system launches read each CTA's descriptor from dSys_
    for (auto const& g : grid_) {
        uint32_t const n = (uint32_t)g.tiles.size();
        cudaError_t err = g.codeMode == kCodeNone ? launch_check(dSys_, g.dTiles, n, kGridBlock, e, stream_)
                                                  : launch_check_bc(unused, dSys_, g.dTiles, n, e, g.codeMode, stream_);
        if (err != cudaSuccess) return err;
        err = g.codeMode == kCodeNone ? launch_perform(dSys_, g.dTiles, n, kGridBlock, e, stream_)
                                      : launch_perform_bc(unused, dSys_, g.dTiles, n, e, g.codeMode, stream_);
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
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
    // every member's own stream must be idle, and pending grid-path marks of members that will
    // run resident must be cleared first
    for (Updater* u : members_) u->synchronize();
    if (!built_) rebuild();
    for (uint32_t m = 0; m < M; ++m)
        if (isResident_[m]) members_[m]->scrubPending(members_[m]->stream());
    for (uint32_t m = 0; m < M; ++m)
        if (isResident_[m]) members_[m]->synchronize();

    std::vector<uint64_t> need(M);
    uint64_t T = 0;
    for (uint32_t m = 0; m < M; ++m) {
        need[m] = (uint64_t)mcs[m] * members_[m]->nColors();
        T = std::max(T, need[m]);
    }
    for (uint64_t t0 = 0; t0 < T; t0 += stepCap_) {
        uint32_t const chunk = (uint32_t)std::min<uint64_t>(stepCap_, T - t0);
        cuda_check(cudaEventSynchronize(stepsFree_), "batch staging");
        for (uint32_t t = 0; t < chunk; ++t)
            for (uint32_t m = 0; m < M; ++m) {
                StepEntry& e = hSteps_[(size_t)t * M + m];
                if (t0 + t < need[m]) e = members_[m]->nextStep();
                else e = StepEntry{kNoColor, 0u, 0u, kNoColor, 0u, 0u, 0u, 0u};
            }
        cuda_check(cudaMemcpyAsync(dSteps_, hSteps_, sizeof(StepEntry) * chunk * M, cudaMemcpyHostToDevice, stream_),
                   "batch steps H2D");
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        if (!resident_.empty()) {
            cuda_check(cudaEventRecord(fork_, stream_), "event");
            cuda_check(cudaStreamWaitEvent(stream2_, fork_, 0), "wait");
            for (auto const& g : resident_) {
                cuda_check(g.codeMode == kCodeNone
                               ? launch_resident(dSys_, g.dList, (uint32_t)g.members.size(), g.perThread, dSteps_, M,
                                                 chunk, g.smem, stream2_)
                               : launch_resident_bc(dSys_, g.dList, (uint32_t)g.members.size(), g.perThread, dSteps_,
                                                    M, chunk, g.smem, g.codeMode, stream2_),
                           "batch resident");
                ++launches_;
            }
        }
        if (!grid_.empty()) {
            if (chunk == stepCap_) {
                if (!graph_) {
                    cudaGraph_t g;
                    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
                    cudaError_t err = cudaSuccess;
                    for (uint32_t t = 0; t < stepCap_ && err == cudaSuccess; ++t) err = launchGrid(t, M);
                    cudaError_t const endErr = cudaStreamEndCapture(stream_, &g);
                    cuda_check(err, "capture batch launches");
                    cuda_check(endErr, "end capture");
                    cudaError_t const ie = cudaGraphInstantiate(&graph_, g, 0);
                    cudaGraphDestroy(g);
                    cuda_check(ie, "graph instantiate");
                }
                cuda_check(cudaGraphLaunch(graph_, stream_), "batch graph launch");
            } else {
                for (uint32_t t = 0; t < chunk; ++t) cuda_check(launchGrid(t, M), "batch grid launch");
            }
            launches_ += 2ull * chunk * grid_.size();
        }
        if (!resident_.empty()) {
            cuda_check(cudaEventRecord(join_, stream2_), "event");
            cuda_check(cudaStreamWaitEvent(stream_, join_, 0), "wait");
        }
    }
    cuda_check(cudaEventRecord(done_, stream_), "event");
    for (uint32_t m = 0; m < M; ++m) {
        members_[m]->noteExternalRun(need[m], (uint64_t)mcs[m], !isResident_[m], members_[m]->lastColor());
        members_[m]->streamWait(done_);
    }
}

float Batch::runTimed(int32_t nMcs)
{
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    for (Updater* u : members_) u->synchronize();
    if (!built_) rebuild();
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
