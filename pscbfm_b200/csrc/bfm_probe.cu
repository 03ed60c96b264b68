// Device probes for the sweep's latency model (bfm_probe_device).
//
// The sweep kernels keep their state (about 40 B per monomer) in the L2 between launches and wait
// on chains of dependent loads, so neither the HBM nor the L2 bandwidth bounds them. What does is
// the latency of one L2 round trip times the dependent round trips of a kernel, plus the time a
// kernel of the sweep's shape takes to launch, spread over the SMs and drain. These probes
// measure both on the device at hand, and the L2's read bandwidth for the bandwidth fraction:
//   - L2 hit latency: one thread follows a random cycle of indices, one per 128-byte line, over a
//     buffer that the L2 holds (loads cached in L2 only), timed by CUDA events over many steps;
//   - L2 read bandwidth: every SM reads a buffer that the L2 holds, 16 bytes per load;
//   - dependent-kernel period: a captured graph of back-to-back kernels of 1024 CTAs x 256
//     threads that do nothing, the floor of a grid-phase launch inside the sweep's graph.

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/bfm.h"

namespace {

__global__ void k_chase(uint32_t const* __restrict__ next, uint32_t steps, uint32_t* sink)
{
    uint32_t i = 0;
    for (uint32_t s = 0; s < steps; ++s) i = __ldcg(next + i);
    *sink = i;
}

__global__ void k_l2_read(uint4 const* __restrict__ buf, size_t n, uint32_t reps, uint32_t* sink)
{
    uint32_t acc = 0;
    size_t const stride = (size_t)gridDim.x * blockDim.x;
    for (uint32_t r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
            uint4 const v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9E3779B9u) *sink = acc;   // keeps the loads; practically never stores
}

__global__ void k_empty() {}

struct Ev {
    cudaEvent_t a = nullptr, b = nullptr;
    Ev()
    {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Ev()
    {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

}  // namespace

extern "C" int bfm_probe_device(int gpu, double out[4])
{
    if (!out) return BFM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(gpu) != cudaSuccess) return BFM_ERR_CUDA;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return BFM_ERR_CUDA;
    uint32_t* chase = nullptr;
    uint4* buf = nullptr;
    uint32_t* sink = nullptr;
    cudaGraphExec_t exec = nullptr;
    int status = BFM_ERR_CUDA;
    do {
        // L2 hit latency: 8 MB, a random cycle through 65,536 lines of 128 bytes
        constexpr uint32_t kLines = 1u << 16, kWordsPerLine = 32, kSteps = 200000;
        std::vector<uint32_t> perm(kLines), next((size_t)kLines * kWordsPerLine, 0u);
        for (uint32_t i = 0; i < kLines; ++i) perm[i] = i;
        uint64_t r = 0x243F6A8885A308D3ull;
        for (uint32_t i = kLines - 1; i > 0; --i) {   // Fisher-Yates with a 64-bit LCG
            r = r * 6364136223846793005ull + 1442695040888963407ull;
            uint32_t const j = (uint32_t)((r >> 33) % (i + 1));
            uint32_t const t = perm[i];
            perm[i] = perm[j];
            perm[j] = t;
        }
        for (uint32_t k = 0; k < kLines; ++k)
            next[(size_t)perm[k] * kWordsPerLine] = perm[(k + 1) % kLines] * kWordsPerLine;
        if (cudaMalloc(&chase, next.size() * 4) != cudaSuccess) break;
        if (cudaMalloc(&sink, 4) != cudaSuccess) break;
        if (cudaMemcpyAsync(chase, next.data(), next.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) break;
        Ev ev;
        k_chase<<<1, 1, 0, s>>>(chase, kLines, sink);   // brings the lines into the L2
        cudaEventRecord(ev.a, s);
        k_chase<<<1, 1, 0, s>>>(chase, kSteps, sink);
        cudaEventRecord(ev.b, s);
        if (cudaEventSynchronize(ev.b) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev.a, ev.b);
        out[0] = ms * 1e6 / kSteps;

        // L2 read bandwidth: 32 MB read 20 times by 8 CTAs of 512 threads per SM
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, gpu);
        constexpr size_t kBytes = 32ull << 20;
        constexpr uint32_t kReps = 20;
        if (cudaMalloc(&buf, kBytes) != cudaSuccess) break;
        if (cudaMemsetAsync(buf, 1, kBytes, s) != cudaSuccess) break;
        k_l2_read<<<nsm * 8, 512, 0, s>>>(buf, kBytes / 16, 1, sink);
        cudaEventRecord(ev.a, s);
        k_l2_read<<<nsm * 8, 512, 0, s>>>(buf, kBytes / 16, kReps, sink);
        cudaEventRecord(ev.b, s);
        if (cudaEventSynchronize(ev.b) != cudaSuccess) break;
        cudaEventElapsedTime(&ms, ev.a, ev.b);
        out[1] = (double)kBytes * kReps / (ms * 1e-3) / 1e9;

        // dependent-kernel period in a captured graph
        constexpr uint32_t kKernels = 200;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) break;
        for (uint32_t k = 0; k < kKernels; ++k) k_empty<<<1024, 256, 0, s>>>();
        if (cudaStreamEndCapture(s, &g) != cudaSuccess) break;
        cudaError_t const ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) break;
        cudaGraphLaunch(exec, s);   // first replay uploads the graph
        cudaEventRecord(ev.a, s);
        cudaGraphLaunch(exec, s);
        cudaEventRecord(ev.b, s);
        if (cudaEventSynchronize(ev.b) != cudaSuccess) break;
        cudaEventElapsedTime(&ms, ev.a, ev.b);
        out[2] = ms * 1e3 / kKernels;
        out[3] = nsm;
        status = BFM_OK;
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    cudaStreamSynchronize(s);
    cudaFree(chase);
    cudaFree(buf);
    cudaFree(sink);
    cudaStreamDestroy(s);
    if (status != BFM_OK) cudaGetLastError();
    return status;
}
