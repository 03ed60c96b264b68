// Batch: many independent systems advanced together on one GPU.
//
// Systems whose three occupancy lattices fit one CTA's shared memory run in the resident kernel,
// one CTA per system, one launch per chunk of sub-steps. The other systems share the grid-phase
// kernels: one check and one perform launch per sub-step cover the active colour group of every
// such system at once, and a chunk of those launches is captured into a CUDA graph once and
// replayed. The two paths run concurrently on two streams. Each system draws its own sub-steps
// from its own stream exactly as it would alone, so its trajectory is unchanged by batching.

#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "bfm_engine.hpp"

namespace bfm {

namespace {
constexpr uint32_t kBatchChunk = 64;      // sub-steps per staged chunk / per captured graph
}

Batch::Batch(int gpu, Updater* const* members, uint32_t n) : gpu_(gpu)
{
    if (n == 0) throw std::invalid_argument("[Batch] no systems");
    for (uint32_t i = 0; i < n; ++i) {
        Updater* u = members[i];
        if (!u) throw std::invalid_argument("[Batch] null system");
        if (!u->initialized()) throw std::runtime_error("[Batch] every system must be initialized");
        if (u->gpu() != gpu) throw std::invalid_argument("[Batch] every system must live on the batch GPU");
        for (uint32_t j = 0; j < i; ++j)
            if (members[j] == u) throw std::invalid_argument("[Batch] a system appears twice");
        members_.push_back(u);
    }
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
    cudaFree(dSys_);
    cudaFreeHost(hSteps_);
    if (join_) cudaEventDestroy(join_);
    if (fork_) cudaEventDestroy(fork_);
    if (stepsFree_) cudaEventDestroy(stepsFree_);
    if (done_) cudaEventDestroy(done_);
    if (stream_) cudaStreamDestroy(stream_);
    if (stream2_) cudaStreamDestroy(stream2_);
}

void Batch::rebuild()
{
    uint32_t const M = (uint32_t)members_.size();
    resident_.clear();
    grid_.clear();
    tiles_.clear();
    residentPerThread_ = 1;
    residentSmem_ = 0;
    for (uint32_t m = 0; m < M; ++m) {
        Updater* u = members_[m];
        if (residentOn_ && u->residentEligible()) {
            resident_.push_back(m);
            SysDev const& d = u->desc();
            residentSmem_ = std::max(residentSmem_, resident_smem_bytes(d.nwords, d.nb[0] + d.nb[1] + d.nb[2]));
            while (residentPerThread_ * kResidentBlock < u->maxGroup()) residentPerThread_ *= 2;
        } else {
            grid_.push_back(m);
            uint32_t const t = std::max((u->maxGroup() + kGridBlock - 1) / kGridBlock, 1u);
            for (uint32_t k = 0; k < t; ++k) tiles_.push_back(TileRef{m, k * kGridBlock});
        }
    }
    stepCap_ = kBatchChunk;
    size_t const stepsBytes = sizeof(StepEntry) * stepCap_ * M;
    size_t const sysBytes = (sizeof(SysDev) * M + 255) & ~size_t(255);
    size_t const tileBytes = (sizeof(TileRef) * std::max<size_t>(tiles_.size(), 1) + 255) & ~size_t(255);
    size_t const listBytes = (sizeof(uint32_t) * std::max<size_t>(resident_.size(), 1) + 255) & ~size_t(255);
    cudaFree(dSys_);
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, sysBytes + tileBytes + listBytes + stepsBytes), "cudaMalloc(batch)");
    char* base = static_cast<char*>(p);
    dSys_ = reinterpret_cast<SysDev*>(base);
    dTiles_ = reinterpret_cast<TileRef*>(base + sysBytes);
    dResList_ = reinterpret_cast<uint32_t*>(base + sysBytes + tileBytes);
    dSteps_ = reinterpret_cast<StepEntry*>(base + sysBytes + tileBytes + listBytes);
    std::vector<SysDev> descs(M);
    for (uint32_t m = 0; m < M; ++m) descs[m] = members_[m]->desc();
    cuda_check(cudaMemcpy(dSys_, descs.data(), sizeof(SysDev) * M, cudaMemcpyHostToDevice), "upload descriptors");
    if (!tiles_.empty())
        cuda_check(cudaMemcpy(dTiles_, tiles_.data(), sizeof(TileRef) * tiles_.size(), cudaMemcpyHostToDevice),
                   "upload tiles");
    if (!resident_.empty())
        cuda_check(cudaMemcpy(dResList_, resident_.data(), sizeof(uint32_t) * resident_.size(), cudaMemcpyHostToDevice),
                   "upload resident list");
    cudaFreeHost(hSteps_);
    hSteps_ = nullptr;
    cuda_check(cudaMallocHost(&hSteps_, stepsBytes), "cudaMallocHost(batch steps)");
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    built_ = true;
}

void Batch::run(int32_t nMcs)
{
    if (nMcs <= 0) return;
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    uint32_t const M = (uint32_t)members_.size();
    // every member's own stream must be idle, and pending grid-path marks of members that will
    // run resident must be cleared first
    for (Updater* u : members_) u->synchronize();
    if (!built_) rebuild();
    for (uint32_t m : resident_) members_[m]->scrubPending(members_[m]->stream());
    for (uint32_t m : resident_) members_[m]->synchronize();

    std::vector<uint64_t> need(M);
    uint64_t T = 0;
    for (uint32_t m = 0; m < M; ++m) {
        need[m] = (uint64_t)nMcs * members_[m]->nColors();
        T = std::max(T, need[m]);
    }
    uint32_t const nGridTiles = (uint32_t)tiles_.size();
    for (uint64_t t0 = 0; t0 < T; t0 += stepCap_) {
        uint32_t const chunk = (uint32_t)std::min<uint64_t>(stepCap_, T - t0);
        cuda_check(cudaEventSynchronize(stepsFree_), "batch staging");
        for (uint32_t t = 0; t < chunk; ++t)
            for (uint32_t m = 0; m < M; ++m) {
                StepEntry& e = hSteps_[(size_t)t * M + m];
                if (t0 + t < need[m]) e = members_[m]->nextStep();
                else e = StepEntry{kNoColor, 0u, 0u, kNoColor};
            }
        cuda_check(cudaMemcpyAsync(dSteps_, hSteps_, sizeof(StepEntry) * chunk * M, cudaMemcpyHostToDevice, stream_),
                   "batch steps H2D");
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        if (!resident_.empty()) {
            cuda_check(cudaEventRecord(fork_, stream_), "event");
            cuda_check(cudaStreamWaitEvent(stream2_, fork_, 0), "wait");
            cuda_check(launch_resident(dSys_, dResList_, (uint32_t)resident_.size(), residentPerThread_, dSteps_, M,
                                       chunk, residentSmem_, stream2_),
                       "batch resident");
        }
        if (nGridTiles) {
            if (chunk == stepCap_) {
                if (!graph_) {
                    cudaGraph_t g;
                    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
                    cudaError_t err = cudaSuccess;
                    for (uint32_t t = 0; t < stepCap_ && err == cudaSuccess; ++t) {
                        err = launch_check(dSys_, dTiles_, nGridTiles, kGridBlock, dSteps_ + (size_t)t * M, stream_);
                        if (err == cudaSuccess)
                            err = launch_perform(dSys_, dTiles_, nGridTiles, kGridBlock, dSteps_ + (size_t)t * M, stream_);
                    }
                    cudaError_t const endErr = cudaStreamEndCapture(stream_, &g);
                    cuda_check(err, "capture batch launches");
                    cuda_check(endErr, "end capture");
                    cudaError_t const ie = cudaGraphInstantiate(&graph_, g, 0);
                    cudaGraphDestroy(g);
                    cuda_check(ie, "graph instantiate");
                }
                cuda_check(cudaGraphLaunch(graph_, stream_), "batch graph launch");
            } else {
                for (uint32_t t = 0; t < chunk; ++t) {
                    cuda_check(launch_check(dSys_, dTiles_, nGridTiles, kGridBlock, dSteps_ + (size_t)t * M, stream_),
                               "batch check");
                    cuda_check(launch_perform(dSys_, dTiles_, nGridTiles, kGridBlock, dSteps_ + (size_t)t * M, stream_),
                               "batch perform");
                }
            }
        }
        if (!resident_.empty()) {
            cuda_check(cudaEventRecord(join_, stream2_), "event");
            cuda_check(cudaStreamWaitEvent(stream_, join_, 0), "wait");
        }
    }
    std::vector<char> isRes(M, 0);
    for (uint32_t m : resident_) isRes[m] = 1;
    cuda_check(cudaEventRecord(done_, stream_), "event");
    for (uint32_t m = 0; m < M; ++m) {
        members_[m]->noteExternalRun(need[m], (uint64_t)nMcs, !isRes[m], members_[m]->lastColor());
        members_[m]->streamWait(done_);
    }
}

float Batch::runTimed(int32_t nMcs)
{
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    for (Updater* u : members_) u->synchronize();
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
