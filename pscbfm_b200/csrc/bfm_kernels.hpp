// Host-callable launchers of the sweep kernels (bfm_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "bfm_device.cuh"

namespace bfm {

constexpr uint32_t kGridBlock = 256;          // threads per CTA of the grid-phase kernels
constexpr uint32_t kResidentBlock = 1024;     // threads per CTA of the resident kernel
// dynamic shared memory of the resident kernel: the 227 KB opt-in limit minus room for its
// static shared memory (the copied system descriptor)
constexpr size_t kResidentMaxSmem = 226 * 1024;
constexpr int32_t kPadCoord = INT32_MIN;      // x of an unused (padding) slot

// One CTA of a grid-phase launch: system index and first in-colour index it covers.
struct TileRef {
    uint32_t sys;
    uint32_t start;
    uint32_t count = 1;   // consecutive tiles from start (bond-code perform lists group up to 4)
};

// dTiles == nullptr: single system 0, CTA b covers [b*tileSpan, (b+1)*tileSpan).
cudaError_t launch_check(SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles, uint32_t tileSpan,
                         StepEntry const* dSteps, cudaStream_t s);
// next != nullptr (one system): CTA 0 writes the following sub-step's entry there (write_next_step)
cudaError_t launch_perform(SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles, uint32_t tileSpan,
                           StepEntry const* dSteps, cudaStream_t s, StepEntry* next = nullptr);

// Resident kernel: CTA b runs system dList[b] through sub-steps 0..nSteps-1 of dSteps
// ([nSteps][nSys] entries). perThread = ceil(largest colour group / kResidentBlock), in {1,2,4,8,16}.
size_t resident_smem_bytes(uint32_t nwords, uint32_t ntab);
cudaError_t launch_resident(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, uint32_t perThread,
                            StepEntry const* dSteps, uint32_t nSys, uint32_t nSteps, size_t smem, cudaStream_t s);

// Bond-code kernels (SysDev::codeMode kCode32 / kCode64). Tiles span kBcTileSpan in-colour
// indices. As in the gather representation, the perform zeroes the previous sub-step's marks, so a
// stand-alone scrub is a perform launch whose entry has color == kNoColor.
constexpr int kCheckMpt = 2;                                   // monomers per thread (256-thread CTAs)
constexpr uint32_t kBcTileSpan = kGridBlock * kCheckMpt;       // 512 in-colour indices per tile
// CTA sizes of the bond-code check: 128, 256 or 512 threads over the same tile (4, 2 or 1
// monomers per thread); every size gives the same results
constexpr uint32_t kCheckBlockDefault = 256;
inline bool check_block_ok(int block) { return block == 128 || block == 256 || block == 512; }
// dTiles == nullptr: single system, descriptor passed by value (hostDesc); otherwise the tile
// list selects the system per CTA from dSys and hostDesc is unused. shape picks the check's register
// budget (resident threads per SM), 0 .. kGridShapes-1, and block its CTA size (check_block_ok);
// negative / 0: the defaults. Every shape and block gives the same results.
constexpr int kGridShapes = 4;
// The perform launch's tile list for a check tile list of bond-code systems: one tile per entry.
std::vector<TileRef> perform_tile_list(std::vector<TileRef> const& tiles);
// snap != nullptr (one system): the check first writes the snapshot of the move counters as the
// work before it left them into that ring (snapshot_stats; the sequence word follows the 4 x
// kSnapRing slot words). The check counts attempted moves (CTA 0, after the snapshot) and the
// perform the tentative ones (list lengths) and the accepted ones.
cudaError_t launch_check_bc(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                            StepEntry const* dSteps, uint32_t codeMode, cudaStream_t s, int shape = -1,
                            int block = 0, unsigned long long* snap = nullptr);
// The perform takes one warp per tile. A single-system launch may carry the sub-step's parity and
// scope (kPerfCur: walk its tentative movers, kPerfPrev: zero the previous sub-step's marks), so
// it reads no step entry; parity == kParityFromEntry reads both from dSteps[0]. next != nullptr
// (one system): CTA 0 writes the following sub-step's entry there (write_next_step). Tile lists
// (several systems) always read each system's entry; parity, scope and next are ignored.
constexpr uint32_t kParityFromEntry = 0xFFFFFFFFu;
constexpr uint32_t kPerformWarpsDefault = 4;   // warps per CTA of the perform
constexpr uint32_t kPerformGroupDefault = 4;   // warps per tile of the perform
// the perform shapes (warps per CTA, warps per tile) an autotuner tries beside the default
constexpr int kPerformShapeTrials[][2] = {{8, 4}, {4, 2}, {8, 8}, {2, 2}};
constexpr uint32_t kPerfCur = 1u, kPerfPrev = 2u;
struct PerformArgs {
    uint32_t parity = kParityFromEntry;
    uint32_t scope = kPerfCur | kPerfPrev;
    StepEntry* next = nullptr;
    unsigned long long* snap = nullptr;   // the check's counter snapshot ring (launch_check_bc)
    int warps = 0;   // warps per CTA (1, 2, 4, 8; 0: the default)
    int group = 0;   // warps per tile (1, 2, 4, 8, at most `warps`; 0: the default)
};
inline bool perform_shape_ok(int warps, int group)
{
    auto ok = [](int v) { return v == 1 || v == 2 || v == 4 || v == 8; };
    return (warps == 0 && group == 0) || (ok(warps) && ok(group) && group <= warps);
}
cudaError_t launch_perform_bc(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                              StepEntry const* dSteps, uint32_t codeMode, cudaStream_t s, int shape = -1,
                              PerformArgs const& pa = PerformArgs{});
// Persistent sweep (bond codes, one system): nSteps sub-steps of check, barrier, perform in one
// launch of at most the co-resident CTA count: a grid of at most 16 CTAs as one thread-block
// cluster (hardware barriers) where allowCluster and the device can run it, otherwise a
// cooperative launch with grid barriers in global memory. gs->count must be zeroed before the
// launch; after it, gs->fault != 0 means a grid-barrier wait ran out and the system's state is not
// usable. shape selects the CTAs per SM the register budget must fit: 0 -> 4, 1 -> 5, 2 -> 6 (two
// monomers per thread, one mover-list segment per tile).
constexpr int kSweepShapes = 3;
cudaError_t launch_sweep_bc(SysDev const& hostDesc, StepEntry const* dSteps, uint32_t nSteps, uint32_t maxGroup,
                            GridSync* gs, uint32_t codeMode, int shape, bool allowCluster, cudaStream_t s,
                            uint32_t* gridOut);
size_t resident_bc_smem_bytes(uint32_t nwords, uint32_t npad, uint32_t maxGroup, uint32_t codeMode);
// Cluster-resident sweep (bond codes): one cluster of 2^logC CTAs of kResidentBlock threads per
// system of dList[0..nClusters) (logC 1..4), state in the cluster's shared memory for nSteps
// sub-steps whose entries are dSteps[t * stride + system]; perThread (1, 2, 4, 8) chunks of 32
// slots per warp and colour. cluster_bc_runnable: whether the device can run that configuration
// (kernel attributes set, cudaOccupancyMaxActiveClusters >= 1).
size_t cluster_bc_smem_bytes(uint32_t nwords, uint32_t npad, uint32_t logC, uint32_t perThread, uint32_t codeMode);
bool cluster_bc_runnable(uint32_t logC, uint32_t perThread, size_t smem, uint32_t codeMode);
cudaError_t launch_cluster_bc(SysDev const* dSys, uint32_t const* dList, uint32_t nClusters, uint32_t logC,
                              uint32_t perThread, StepEntry const* dSteps, uint32_t stride, uint32_t nSteps,
                              size_t smem, uint32_t codeMode, cudaStream_t s);
cudaError_t launch_resident_bc(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, uint32_t perThread,
                               StepEntry const* dSteps, uint32_t nSys, uint32_t nSteps, size_t smem, uint32_t codeMode,
                               cudaStream_t s);

// Observables (bfm_observables.cu). Molecule of every slot (kNoColor for padding), first and last
// slot of every molecule, and the reference positions for the mean squared displacement.
struct ObsDev {
    uint32_t const* molOfSlot;
    uint32_t const* ends;       // [2 * nMol]
    int32_t const* rx;
    int32_t const* ry;
    int32_t const* rz;
    uint32_t nMol;
};
inline size_t obs_words(uint32_t nMol) { return 5ull * nMol + 512 + 1; }
cudaError_t launch_observables(SysDev const* dSys, ObsDev const& o, long long* dOut, uint32_t npad, cudaStream_t s);

// Sets the occupancy bit of every non-padding slot of system dSys[0] (lat must be zeroed).
cudaError_t launch_build_lattice(SysDev const* dSys, uint32_t npad, cudaStream_t s);
// Positions in the caller's order, x y z interleaved (out[3 i + a] from sorted slot slotOf[i]).
cudaError_t launch_gather_positions(SysDev const& h, uint32_t const* slotOf, uint32_t n, int32_t* out,
                                    cudaStream_t s);
// Unfolded positions of every slot of bond-code system dSys[0] (image offsets plus the coordinates
// of the lattice addresses) into ox, oy, oz, in slot order.
cudaError_t launch_unfold_positions(SysDev const* dSys, uint32_t npad, int32_t* ox, int32_t* oy, int32_t* oz,
                                    cudaStream_t s);
// Writes the sums over the kStatSlots slots of the three move counters (attempted, tentative,
// accepted) into out[0..3), mapped pinned host memory.
cudaError_t launch_publish_stats(unsigned long long const* stats, unsigned long long* out, cudaStream_t s);
// A counter snapshot (snapshot_stats) as a one-warp launch: a captured sweep graph's last node
// when its handle's counters are read by ticket; k_publish_snap copies one slot of the snapshot
// ring into host memory, on another stream.
cudaError_t launch_snapshot_stats(unsigned long long const* stats, unsigned long long* ring, unsigned long long* seq,
                                  cudaStream_t s);
cudaError_t launch_publish_snap(unsigned long long const* slot, unsigned long long* out, cudaStream_t s);

}  // namespace bfm
