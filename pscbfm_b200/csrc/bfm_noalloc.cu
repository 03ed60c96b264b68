// Sweep entry point that allocates nothing.
//
// Some callers cannot let a library allocate device memory: a host program that has already
// reserved the GPU's memory for its own pool (a simulation framework with its own allocator, or a
// serving process that claimed its HBM budget at start-up), and latency-sensitive loops where a
// cudaMalloc/cudaFree pair would synchronise the device in the middle of a run. For them,
// bfm_sweep_noalloc runs the same grid-phase check/perform kernels as bfm_run on buffers the
// caller owns; the engine's per-sub-step scratch (tentative flags, temporary-lattice marks, the
// two temporary lattices, the occupancy lattice, brick tables, the descriptor and the sub-step
// entries) lives in one file-scope device array of kScratchBytes, which every GPU that loads
// the library holds until the process exits.
//
// Set-up: the first call on a device (with that device current) looks the array's device
// address up once with cudaGetSymbolAddress; make that first call before any stream capture.
// Every call shares the array and overwrites what the previous call left there, so calls that
// overlap on the GPU (two streams, two threads) race: serialise them.

#include <cuda_runtime.h>

#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/bfm.h"
#include "bfm_device.cuh"
#include "bfm_kernels.hpp"

namespace {

constexpr size_t kScratchBytes = 32ull << 20;       // 32 MiB, shared by every call
constexpr uint32_t kStepRing = 4096;                 // sub-step entries staged per copy
constexpr uint32_t kHostChunk = 256;                 // entries built on the host stack per copy
constexpr uint32_t kMaxBricksPerAxis = 256;          // box sides up to 1024

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex gSetupMutex;
void* gScratchAddr[64] = {};

size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

int fail(char* err, size_t len, int code, char const* fmt, ...)
{
    if (err && len) {
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(err, len, fmt, ap);
        va_end(ap);
    }
    return code;
}

uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint32_t draw(uint64_t seed, uint64_t k) { return (uint32_t)(mix64(mix64(seed) + (k + 1) * 0x9E3779B97F4A7C15ull) >> 32); }

}  // namespace

extern "C" int bfm_sweep_noalloc(const bfm_noalloc_system* s, int32_t n_mcs, uint64_t seed, uint64_t substep0,
                                 void* stream_ptr, char* err, size_t err_len)
{
    using namespace bfm;
    if (!s || !s->x || !s->y || !s->z || !s->nbr || !s->nnb || !s->group_offset || !s->group_size || !s->forbidden)
        return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT, "[bfm_sweep_noalloc] null pointer in the system");
    if (n_mcs < 0) return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT, "[bfm_sweep_noalloc] negative MCS count");
    uint32_t const nC = s->n_colors;
    if (nC == 0 || nC > 255 || s->npad == 0 || s->maxc == 0 || s->maxc > (uint32_t)kMaxConn)
        return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT,
                    "[bfm_sweep_noalloc] need 1..255 colours, npad > 0 and 1..%d neighbour slots", kMaxConn);
    for (int a = 0; a < 3; ++a) {
        uint32_t const b = s->box[a];
        if (b < 4 || b > 4 * kMaxBricksPerAxis || (b & (b - 1)))
            return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT,
                        "[bfm_sweep_noalloc] box sides must be powers of two in [4, 1024]");
    }
    uint32_t maxGroup = 0;
    for (uint32_t c = 0; c < nC; ++c) {
        if ((uint64_t)s->group_offset[c] + s->group_size[c] > s->npad)
            return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT, "[bfm_sweep_noalloc] colour group %u exceeds npad", c);
        if (s->group_size[c] > maxGroup) maxGroup = s->group_size[c];
    }
    uint32_t nb[3] = {s->box[0] / 4, s->box[1] / 4, s->box[2] / 4};
    uint64_t const nwords = (uint64_t)nb[0] * nb[1] * nb[2];
    uint32_t const ntab = nb[0] + nb[1] + nb[2];

    // scratch layout
    size_t const oDesc = 0;
    size_t const oSteps = up256(oDesc + sizeof(SysDev));
    size_t const oGrp = up256(oSteps + sizeof(StepEntry) * kStepRing);
    size_t const oTab = up256(oGrp + sizeof(uint32_t) * 2 * 255);
    size_t const oStats = up256(oTab + sizeof(uint32_t) * 3 * kMaxBricksPerAxis);
    size_t const oFlags = up256(oStats + kStatBytes);
    size_t const oMark = up256(oFlags + (size_t)s->npad);
    size_t const oLat = up256(oMark + 8ull * s->npad);
    size_t const oTmp = up256(oLat + 8ull * nwords);
    size_t const need = up256(oTmp + 16ull * nwords);
    if (need > kScratchBytes)
        return fail(err, err_len, BFM_ERR_INVALID_ARGUMENT,
                    "[bfm_sweep_noalloc] system needs %zu bytes of scratch, the fixed array holds %zu (32 MiB)", need,
                    kScratchBytes);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return fail(err, err_len, BFM_ERR_CUDA, "[bfm_sweep_noalloc] cudaGetDevice: %s", cudaGetErrorString(e));
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(gSetupMutex);
        if (!gScratchAddr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess || !p)
                return fail(err, err_len, BFM_ERR_CUDA, "[bfm_sweep_noalloc] cudaGetSymbolAddress: %s",
                            cudaGetErrorString(e));
            gScratchAddr[dev] = p;
        }
        base = gScratchAddr[dev];
    }
    char* const B = static_cast<char*>(base);
    cudaStream_t const st = static_cast<cudaStream_t>(stream_ptr);

    // descriptor (host stack copy), group table, brick tables; every axis is periodic (walls = 0)
    SysDev d;
    std::memset(&d, 0, sizeof(d));
    d.x = s->x;
    d.y = s->y;
    d.z = s->z;
    d.nbr = s->nbr;
    d.nnb = s->nnb;
    d.flags = reinterpret_cast<uint8_t*>(B + oFlags);
    d.tmark = reinterpret_cast<uint32_t*>(B + oMark);
    d.lat = reinterpret_cast<unsigned long long*>(B + oLat);
    d.tmp = reinterpret_cast<unsigned long long*>(B + oTmp);
    d.brickTab = reinterpret_cast<uint32_t*>(B + oTab);
    d.grp = reinterpret_cast<uint32_t*>(B + oGrp);
    d.stats = reinterpret_cast<unsigned long long*>(B + oStats);
    d.npad = s->npad;
    d.nwords = (uint32_t)nwords;
    d.maxc = s->maxc;
    d.nColors = nC;
    for (int a = 0; a < 3; ++a) {
        d.mask[a] = s->box[a] - 1;
        d.lim[a] = s->box[a] - 1;
        d.nb[a] = nb[a];
    }
    for (uint32_t i = 0; i < 512; ++i)
        if (s->forbidden[i]) d.forbid[i >> 5] |= 1u << (i & 31);

    uint32_t grp[2 * 255];
    for (uint32_t c = 0; c < nC; ++c) {
        grp[2 * c] = s->group_offset[c];
        grp[2 * c + 1] = s->group_size[c];
    }
    uint32_t tab[3 * kMaxBricksPerAxis];
    brick_tables_fill(nb, tab);
    brick_params(nb, d.mb, d.hx, d.hy);
    SysDev* const dDesc = reinterpret_cast<SysDev*>(B + oDesc);
    StepEntry* const dSteps = reinterpret_cast<StepEntry*>(B + oSteps);
#define NOALLOC_CHECK(call, what)                                                                      \
    do {                                                                                               \
        cudaError_t const ce = (call);                                                                 \
        if (ce != cudaSuccess) {                                                                       \
            cudaGetLastError();                                                                        \
            return fail(err, err_len, BFM_ERR_CUDA, "[bfm_sweep_noalloc] %s: %s", what, cudaGetErrorString(ce)); \
        }                                                                                              \
    } while (0)
    // host sources are stack memory: these copies are staged before the calls return
    NOALLOC_CHECK(cudaMemcpyAsync(dDesc, &d, sizeof(SysDev), cudaMemcpyHostToDevice, st), "descriptor copy");
    NOALLOC_CHECK(cudaMemcpyAsync(B + oGrp, grp, sizeof(uint32_t) * 2 * nC, cudaMemcpyHostToDevice, st), "group copy");
    NOALLOC_CHECK(cudaMemcpyAsync(B + oTab, tab, sizeof(uint32_t) * ntab, cudaMemcpyHostToDevice, st), "brick table copy");
    // what must start at zero: counters, both temporary lattices, the occupancy lattice (rebuilt
    // from the caller's positions)
    NOALLOC_CHECK(cudaMemsetAsync(B + oStats, 0, kStatBytes, st), "clear counters");
    NOALLOC_CHECK(cudaMemsetAsync(B + oTmp, 0, 16ull * nwords, st), "clear temporary lattices");
    NOALLOC_CHECK(cudaMemsetAsync(B + oLat, 0, 8ull * nwords, st), "clear lattice");
    NOALLOC_CHECK(launch_build_lattice(dDesc, s->npad, st), "build lattice");

    uint32_t const tiles = maxGroup ? (maxGroup + kGridBlock - 1) / kGridBlock : 1u;
    uint64_t const total = (uint64_t)n_mcs * nC;
    uint32_t last = kNoColor;
    StepEntry chunk[kHostChunk];
    uint32_t ring = 0;
    for (uint64_t t = 0; t < total;) {
        uint32_t const m = (uint32_t)((total - t) < kHostChunk ? (total - t) : kHostChunk);
        // Reusing the ring from its start needs no wait: the copy below is queued on the same
        // stream as the kernels that read the old entries, so it runs after them, and the host
        // chunk is staged before cudaMemcpyAsync returns.
        if (ring + m > kStepRing) ring = 0;
        for (uint32_t i = 0; i < m; ++i) {
            uint64_t const sub = substep0 + t + i;
            StepEntry& q = chunk[i];
            q.color = draw(seed, 2 * sub) % nC;
            q.seed = draw(seed, 2 * sub + 1);
            q.parity = (uint32_t)(sub & 1u);
            q.prevColor = last;
            q.off = s->group_offset[q.color];
            q.cnt = s->group_size[q.color];
            q.poff = last == kNoColor ? 0u : s->group_offset[last];
            q.pcnt = last == kNoColor ? 0u : s->group_size[last];
            last = q.color;
        }
        NOALLOC_CHECK(cudaMemcpyAsync(dSteps + ring, chunk, sizeof(StepEntry) * m, cudaMemcpyHostToDevice, st),
                      "sub-step copy");
        for (uint32_t i = 0; i < m; ++i) {
            NOALLOC_CHECK(launch_check(dDesc, nullptr, tiles, kGridBlock, dSteps + ring + i, st), "check launch");
            NOALLOC_CHECK(launch_perform(dDesc, nullptr, tiles, kGridBlock, dSteps + ring + i, st), "perform launch");
        }
        ring += m;
        t += m;
    }
#undef NOALLOC_CHECK
    return BFM_OK;
}
