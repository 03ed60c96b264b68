// ORACLE PIN — TEST INFRASTRUCTURE ONLY.
//
// Drives pscbfm's own GPU updater, compiled for sm_100a from the reference sources by
// oracle/Makefile (target `ref`, outputs oracle/_ref/libpscbfm_ref*.so), through its setter API in
// the order GPUScBFM_AB_Type::initialize/execute use (src/pscbfm/GPUScBFM_AB_Type.h:78-163).
// The GPU tests call it to pin the CPU oracle (oracle/bfm_oracle.cpp) and the engine against the
// reference kernels on identical inputs and an identical host draw stream; bench.py's
// reference-updater leg times it (bfmref_time) on the same device as the engine.

#include <cstdint>
#include <cstdio>
#include <chrono>
#include <exception>
#include <string>

#include "UpdaterGPUScBFM_AB_Type.h"

#ifdef BFMREF_MAX_CONNECTIVITY
static_assert(MAX_CONNECTIVITY == BFMREF_MAX_CONNECTIVITY, "the harness must see the patched header");
#endif

namespace {
uint32_t const* gDraws = nullptr;
uint64_t gLen = 0, gPos = 0;
bool gShort = false;

// The setter sequence of GPUScBFM_AB_Type::initialize (GPUScBFM_AB_Type.h:78-136) up to and
// including initialize().
void setup(UpdaterGPUScBFM_AB_Type& u, uint32_t n, int32_t const* xyz, uint32_t const* nbrCount,
           uint32_t const* nbrIds, uint32_t maxc, uint32_t const* box, uint8_t const* forbidden)
{
#ifdef NONPERIODICITY
    u.setPeriodicity(false, false, false);   // the only choice this build accepts
#else
    u.setPeriodicity(true, true, true);
#endif
    u.setNrOfAllMonomers(n);
    for (uint32_t i = 0; i < n; ++i) u.setMonomerCoordinates(i, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    for (uint32_t i = 0; i < n; ++i) u.setAttribute(i, 1);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < nbrCount[i]; ++j) u.setConnectivity(i, nbrIds[(size_t)i * maxc + j]);
    u.setLatticeSize(box[0], box[1], box[2]);
    u.populateLattice();
    for (int dx = -4; dx < 4; ++dx)
        for (int dy = -4; dy < 4; ++dy)
            for (int dz = -4; dz < 4; ++dz) {
                uint32_t const idx = (uint32_t(dx) & 7u) | ((uint32_t(dy) & 7u) << 3) | ((uint32_t(dz) & 7u) << 6);
                u.copyBondSet(dx, dy, dz, forbidden[idx] != 0);
            }
    u.initialize();
}

void read_back(UpdaterGPUScBFM_AB_Type& u, uint32_t n, int32_t* xyzOut)
{
    for (uint32_t i = 0; i < n; ++i) {
        xyzOut[3 * i] = u.getMonomerPositionInX(i);
        xyzOut[3 * i + 1] = u.getMonomerPositionInY(i);
        xyzOut[3 * i + 2] = u.getMonomerPositionInZ(i);
    }
}

// setGpu (UpdaterGPUScBFM_AB_Type.cu:472-487) prints the device properties first, and that printer
// builds a std::string from getCudaCodeName(), which returns 0 for any compute capability above 7
// (src/pscbfm/cudacommon.hpp:835-849) and so throws on a B200. The device is selected directly
// instead; initialize() reads it back with cudaGetDevice.
bool select_device(int gpu, char* err, int errLen)
{
    if (cudaSetDevice(gpu) != cudaSuccess) {
        std::snprintf(err, (size_t)errLen, "cudaSetDevice(%d) failed", gpu);
        return false;
    }
    return true;
}
}  // namespace

extern "C" uint32_t bfmref_next_draw(void)
{
    if (gPos < gLen) return gDraws[gPos++];
    gShort = true;
    return 0;
}

// The MAX_CONNECTIVITY this library was compiled with (bonds per monomer it accepts).
extern "C" int bfmref_max_connectivity(void) { return MAX_CONNECTIVITY; }

extern "C" int bfmref_run(int gpu, uint32_t n, int32_t const* xyz, uint32_t const* nbrCount,
                          uint32_t const* nbrIds, uint32_t maxc, uint32_t const* box,
                          uint8_t const* forbidden, uint32_t const* draws, uint64_t nDraws,
                          uint32_t const* chunks, uint32_t nChunks, int32_t* xyzOut,
                          uint64_t* drawsUsed, char* err, int errLen)
{
    try {
        if (!select_device(gpu, err, errLen)) return -1;
        UpdaterGPUScBFM_AB_Type u;
        setup(u, n, xyz, nbrCount, nbrIds, maxc, box, forbidden);
        gDraws = draws;
        gLen = nDraws;
        gPos = 0;
        gShort = false;
        for (uint32_t c = 0; c < nChunks; ++c) u.runSimulationOnGPU((int32_t)chunks[c]);
        read_back(u, n, xyzOut);
        u.cleanup();
        if (drawsUsed) *drawsUsed = gPos;
        if (gShort) {
            std::snprintf(err, (size_t)errLen, "draw list exhausted after %llu draws", (unsigned long long)gLen);
            return -2;
        }
        return 0;
    } catch (std::exception const& e) {
        std::snprintf(err, (size_t)errLen, "%s", e.what());
        return -1;
    }
}

// Times the reference updater on one system: after initialize(), one untimed call of warmMcs MCS,
// then `reps` calls of runSimulationOnGPU(timedMcs). Each timed call is bracketed by CUDA events on
// the legacy default stream, the stream the updater runs on (mStream = 0,
// UpdaterGPUScBFM_AB_Type.cu:417), as its own tGpuLoop figure is (CRITICAL.cu:492-498, :656-666);
// the call also copies the positions back and un-sorts them on the host (CRITICAL.cu:668-697),
// which the host clock (wallS, the reference's MCS*N/t, CRITICAL.cu:679-682) includes and the
// device time (gpuMs) includes up to the copy. Outputs are sums over the timed calls.
extern "C" int bfmref_time(int gpu, uint32_t n, int32_t const* xyz, uint32_t const* nbrCount,
                           uint32_t const* nbrIds, uint32_t maxc, uint32_t const* box,
                           uint8_t const* forbidden, uint32_t const* draws, uint64_t nDraws,
                           uint32_t warmMcs, uint32_t timedMcs, uint32_t reps, float* gpuMs, double* wallS,
                           int32_t* xyzOut, char* err, int errLen)
{
    try {
        if (!select_device(gpu, err, errLen)) return -1;
        UpdaterGPUScBFM_AB_Type u;
        setup(u, n, xyz, nbrCount, nbrIds, maxc, box, forbidden);
        gDraws = draws;
        gLen = nDraws;
        gPos = 0;
        gShort = false;
        if (warmMcs) u.runSimulationOnGPU((int32_t)warmMcs);
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
            std::snprintf(err, (size_t)errLen, "cudaEventCreate failed");
            return -1;
        }
        float ms = 0.f;
        double wall = 0.0;
        for (uint32_t r = 0; r < reps; ++r) {
            cudaDeviceSynchronize();
            auto const t0 = std::chrono::steady_clock::now();
            cudaEventRecord(a, 0);
            u.runSimulationOnGPU((int32_t)timedMcs);
            cudaEventRecord(b, 0);
            auto const t1 = std::chrono::steady_clock::now();
            cudaEventSynchronize(b);
            float m = 0.f;
            cudaEventElapsedTime(&m, a, b);
            ms += m;
            wall += std::chrono::duration<double>(t1 - t0).count();
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaError_t const e = cudaGetLastError();
        if (e != cudaSuccess) {
            std::snprintf(err, (size_t)errLen, "CUDA error: %s", cudaGetErrorString(e));
            return -1;
        }
        if (xyzOut) read_back(u, n, xyzOut);
        u.cleanup();
        *gpuMs = ms;
        *wallS = wall;
        if (gShort) {
            std::snprintf(err, (size_t)errLen, "draw list exhausted after %llu draws", (unsigned long long)gLen);
            return -2;
        }
        return 0;
    } catch (std::exception const& e) {
        std::snprintf(err, (size_t)errLen, "%s", e.what());
        return -1;
    }
}
