// bfm_lemonade.hpp — LeMonADE updater over the B200 engine: the counterpart of pscbfm's adapter
// GPUScBFM_AB_Type<Ingredients> (src/pscbfm/GPUScBFM_AB_Type.h:22-196), for programs that build
// their system with LeMonADE (Ingredients, FeatureMoleculesIO, analyzers) and hand the sweep to the
// GPU. It needs LeMonADE's headers (AbstractUpdater, VectorInt3) and links against libbfm.so.
//
//     UpdaterB200ScBFM<Ing> gpu(ingredients, nMcsPerCall, iGpu);   // same arguments as the
//     taskManager.addUpdater(&gpu);                                // reference adapter
//
// initialize() copies the system from the ingredients into the engine in one bulk call per kind
// of data (positions, attributes, bonds in LeMonADE's neighbour order, box, periodicity, the bond
// set over [-4,3]^3); execute() runs nMcsPerCall MCS, copies the positions back into the molecules
// and advances their age; cleanup() frees the device state. The ingredient calls are the ones the
// reference adapter makes (GPUScBFM_AB_Type.h:78-176), since they are LeMonADE's interface.
//
// Random stream: by default the engine's counter stream with the seed given to setSeed() (0
// unless set). To drive the sweep with LeMonADE's own generator, pass a draw function to
// setDrawCallback() before initialize(), e.g. one that returns rng.r250_rand32().
#pragma once

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <LeMonADE/updater/AbstractUpdater.h>
#include <LeMonADE/utility/Vector3D.h>

#include "bfm_updater.hpp"

template <class T_IngredientsType>
class UpdaterB200ScBFM : public AbstractUpdater
{
public:
    typedef T_IngredientsType IngredientsType;
    typedef typename T_IngredientsType::molecules_type MoleculesType;

    UpdaterB200ScBFM(T_IngredientsType& ingredients, uint32_t nMcsPerCall, int iGpu = 0)
        : ingredients_(ingredients), molecules_(ingredients.modifyMolecules()), nMcs_(nMcsPerCall), gpu_(iGpu)
    {
    }

    void setSeed(uint64_t seed) { seed_ = seed; }
    void setDrawCallback(bfm_draw_fn fn, void* ctx)
    {
        drawFn_ = fn;
        drawCtx_ = ctx;
    }

    void initialize()
    {
        auto const t0 = std::chrono::steady_clock::now();
        bfm_handle const h = updater_.handle();
        updater_.setGpu(gpu_);
        updater_.setPeriodicity(ingredients_.isPeriodicX(), ingredients_.isPeriodicY(), ingredients_.isPeriodicZ());
        uint32_t const n = (uint32_t)ingredients_.getMolecules().size();
        updater_.setNrOfAllMonomers(n);
        std::vector<int32_t> xyz(3ull * n), attr(n);
        std::vector<uint32_t> pairs;
        for (uint32_t i = 0; i < n; ++i) {
            xyz[3ull * i] = (int32_t)molecules_[i].getX();
            xyz[3ull * i + 1] = (int32_t)molecules_[i].getY();
            xyz[3ull * i + 2] = (int32_t)molecules_[i].getZ();
            attr[i] = (int32_t)ingredients_.getMolecules()[i].getAttributeTag();
            // every directed link in LeMonADE's order: the engine's colouring follows list order
            for (std::size_t k = 0; k < ingredients_.getMolecules().getNumLinks(i); ++k) {
                pairs.push_back(i);
                pairs.push_back((uint32_t)ingredients_.getMolecules().getNeighborIdx(i, k));
            }
        }
        check(bfm_set_coords_bulk(h, xyz.data(), n));
        check(bfm_set_attributes_bulk(h, attr.data(), n));
        check(bfm_add_bonds_bulk(h, pairs.data(), (uint32_t)(pairs.size() / 2)));
        updater_.setLatticeSize(ingredients_.getBoxX(), ingredients_.getBoxY(), ingredients_.getBoxZ());
        updater_.populateLattice();
        for (int dx = -4; dx < 4; ++dx)
            for (int dy = -4; dy < 4; ++dy)
                for (int dz = -4; dz < 4; ++dz)
                    updater_.copyBondSet(dx, dy, dz, !ingredients_.getBondset().isValid(VectorInt3(dx, dy, dz)));
        if (drawFn_) updater_.setDrawCallback(drawFn_, drawCtx_);
        else updater_.setSeed(seed_);
        updater_.initialize();
        initSeconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    bool execute()
    {
        auto const t0 = std::chrono::steady_clock::now();
        updater_.runSimulationOnGPU((int32_t)nMcs_);
        uint32_t const n = (uint32_t)ingredients_.getMolecules().size();
        std::vector<int32_t> xyz(3ull * n);
        check(bfm_get_coords_bulk(updater_.handle(), xyz.data(), n));
        for (uint32_t i = 0; i < n; ++i)
            molecules_[i].setAllCoordinates(xyz[3ull * i], xyz[3ull * i + 1], xyz[3ull * i + 2]);
        ingredients_.modifyMolecules().setAge(ingredients_.modifyMolecules().getAge() + nMcs_);
        double const dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        lastMovesPerSecond_ = dt > 0 ? (double)nMcs_ * (double)n / dt : 0.0;
        return true;
    }

    void cleanup() { updater_.cleanup(); }

    double initSeconds() const { return initSeconds_; }
    // attempted moves per second of the last execute(), positions copied back included
    double lastMovesPerSecond() const { return lastMovesPerSecond_; }
    UpdaterGPUScBFM_AB_Type& engine() { return updater_; }

private:
    void check(int status)
    {
        if (status != BFM_OK) throw std::runtime_error(bfm_last_error(updater_.handle()));
    }

    T_IngredientsType& ingredients_;
    MoleculesType& molecules_;
    uint32_t nMcs_;
    int gpu_;
    uint64_t seed_ = 0;
    bfm_draw_fn drawFn_ = nullptr;
    void* drawCtx_ = nullptr;
    UpdaterGPUScBFM_AB_Type updater_;
    double initSeconds_ = 0.0, lastMovesPerSecond_ = 0.0;
};
