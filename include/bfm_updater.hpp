// bfm_updater.hpp — header-only C++ class with the reference's name and methods over the C-ABI
// (include/bfm.h), so callers written against pscbfm's UpdaterGPUScBFM_AB_Type
// (src/pscbfm/UpdaterGPUScBFM_AB_Type.h:316-358; caller: src/pscbfm/GPUScBFM_AB_Type.h:78-196)
// compile unchanged. Non-zero status codes become the reference's exception types.
#pragma once

#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "bfm.h"

class UpdaterGPUScBFM_AB_Type
{
public:
    UpdaterGPUScBFM_AB_Type() { check(bfm_create(&h_, 0), nullptr); }
    virtual ~UpdaterGPUScBFM_AB_Type() { bfm_destroy(h_); }
    UpdaterGPUScBFM_AB_Type(UpdaterGPUScBFM_AB_Type const&) = delete;
    UpdaterGPUScBFM_AB_Type& operator=(UpdaterGPUScBFM_AB_Type const&) = delete;

    void initialize() { check(bfm_initialize(h_)); }
    bool execute() { return true; }
    void cleanup() { check(bfm_cleanup(h_)); }
    void destruct() { check(bfm_cleanup(h_)); }

    void setGpu(int iGpuToUse) { check(bfm_set_gpu(h_, iGpuToUse)); }
    void copyBondSet(int dx, int dy, int dz, bool bondForbidden)
    {
        check(bfm_set_bond_forbidden(h_, dx, dy, dz, bondForbidden ? 1 : 0));
    }
    void setNrOfAllMonomers(uint32_t n) { check(bfm_set_n_monomers(h_, n)); }
    void setAttribute(uint32_t i, int32_t attribute) { check(bfm_set_attribute(h_, i, attribute)); }
    void setMonomerCoordinates(uint32_t i, int32_t x, int32_t y, int32_t z) { check(bfm_set_coords(h_, i, x, y, z)); }
    void setConnectivity(uint32_t a, uint32_t b) { check(bfm_add_bond(h_, a, b)); }
    void setLatticeSize(uint32_t bx, uint32_t by, uint32_t bz) { check(bfm_set_box(h_, bx, by, bz)); }
    void populateLattice() { check(bfm_populate_lattice(h_)); }
    void runSimulationOnGPU(int32_t nMcs)
    {
        check(bfm_run(h_, nMcs));
        mtCopyBack0 = std::chrono::high_resolution_clock::now();
    }
    int32_t getMonomerPositionInX(uint32_t i) { return coord(i, 0); }
    int32_t getMonomerPositionInY(uint32_t i) { return coord(i, 1); }
    int32_t getMonomerPositionInZ(uint32_t i) { return coord(i, 2); }
    void setPeriodicity(bool px, bool py, bool pz) { check(bfm_set_periodicity(h_, px, py, pz)); }

    // when the last runSimulationOnGPU finished its sweep, before the positions are read back
    // (the reference's public member, CRITICAL.cu:656, which its adapter reads)
    std::chrono::time_point<std::chrono::high_resolution_clock> mtCopyBack0;

    // engine extensions
    void setSeed(uint64_t seed) { check(bfm_set_seed(h_, seed)); }
    void setDrawCallback(bfm_draw_fn fn, void* ctx) { check(bfm_set_draw_callback(h_, fn, ctx)); }
    bfm_handle handle() const { return h_; }

private:
    int32_t coord(uint32_t i, int axis)
    {
        int32_t v = 0;
        check(bfm_get_coord(h_, i, axis, &v));
        return v;
    }
    void check(int status) { check(status, h_); }
    static void check(int status, bfm_handle h)
    {
        if (status == BFM_OK) return;
        std::string const msg = bfm_last_error(h);
        switch (status) {
        case BFM_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
        case BFM_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
        default: throw std::runtime_error(msg);
        }
    }
    bfm_handle h_ = nullptr;
};
