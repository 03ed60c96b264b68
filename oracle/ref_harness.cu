// ORACLE PIN — TEST INFRASTRUCTURE ONLY.
//
// Drives pscbfm's own GPU updater, compiled for sm_100a from the reference sources by
// oracle/Makefile (target `ref`, output oracle/_ref/libpscbfm_ref.so), through its setter API in
// the order GPUScBFM_AB_Type::initialize/execute use (src/pscbfm/GPUScBFM_AB_Type.h:78-163).
// The GPU tests call it to pin the CPU oracle (oracle/bfm_oracle.cpp) against the
// reference kernels on identical inputs and an identical host draw stream.

#include <cstdint>
#include <cstdio>
#include <exception>
#include <string>

#include "UpdaterGPUScBFM_AB_Type.h"

namespace {
uint32_t const* gDraws = nullptr;
uint64_t gLen = 0, gPos = 0;
bool gShort = false;
}  // namespace

extern "C" uint32_t bfmref_next_draw(void)
{
    if (gPos < gLen) return gDraws[gPos++];
    gShort = true;
    return 0;
}

extern "C" int bfmref_run(int gpu, uint32_t n, int32_t const* xyz, uint32_t const* nbrCount,
                          uint32_t const* nbrIds, uint32_t maxc, uint32_t const* box,
                          uint8_t const* forbidden, uint32_t const* draws, uint64_t nDraws,
                          uint32_t const* chunks, uint32_t nChunks, int32_t* xyzOut,
                          uint64_t* drawsUsed, char* err, int errLen)
{
    try {
        // setGpu (UpdaterGPUScBFM_AB_Type.cu:472-487) prints the device properties first, and that
        // printer builds a std::string from getCudaCodeName(), which returns 0 for any compute
        // capability above 7 (src/pscbfm/cudacommon.hpp:835-849) and so throws on a B200. The
        // device is selected directly instead; initialize() reads it back with cudaGetDevice.
        if (cudaSetDevice(gpu) != cudaSuccess) {
            std::snprintf(err, (size_t)errLen, "cudaSetDevice(%d) failed", gpu);
            return -1;
        }
        UpdaterGPUScBFM_AB_Type u;
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
        gDraws = draws;
        gLen = nDraws;
        gPos = 0;
        gShort = false;
        for (uint32_t c = 0; c < nChunks; ++c) u.runSimulationOnGPU((int32_t)chunks[c]);
        for (uint32_t i = 0; i < n; ++i) {
            xyzOut[3 * i] = u.getMonomerPositionInX(i);
            xyzOut[3 * i + 1] = u.getMonomerPositionInY(i);
            xyzOut[3 * i + 2] = u.getMonomerPositionInZ(i);
        }
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
