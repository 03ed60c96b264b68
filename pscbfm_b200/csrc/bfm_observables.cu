// int64 observables of one system, exact (no floating point on the device).
//
// Output layout (int64, nMol molecules = connected components of the bond graph, numbered in
// order of their lowest monomer id):
//   [0, 4 nMol)            per molecule: sum x, sum y, sum z, sum (x^2 + y^2 + z^2)
//   [4 nMol, 5 nMol)       per molecule: |r_last - r_first|^2 (lowest and highest monomer id)
//   [5 nMol, 5 nMol + 512) bond-vector histogram by bond-table index (every listed bond entry)
//   [5 nMol + 512]         sum over monomers of |r - r_ref|^2 (r_ref: positions at the last reset)
// Rg^2 of molecule m with n_m monomers = S2/n_m - |S1|^2/n_m^2; the host converts.
// The reference has no observables on the device (analysis lived in LeMonADE); the CPU oracle is a
// plain int64 recomputation from the positions.

#include <cuda_runtime.h>

#include <cstdint>

#include "bfm_device.cuh"
#include "bfm_kernels.hpp"

namespace bfm {

__global__ void __launch_bounds__(256) k_observables(SysDev const* __restrict__ sysv, ObsDev const o,
                                                     long long* __restrict__ out)
{
    __shared__ unsigned int hist[512];
    __shared__ long long msd;
    SysDev const& S = sysv[0];
    for (uint32_t b = threadIdx.x; b < 512; b += blockDim.x) hist[b] = 0;
    if (threadIdx.x == 0) msd = 0;
    __syncthreads();
    long long* const mom = out;
    long long* const ree = out + 4ull * o.nMol;
    long long* const gh = out + 5ull * o.nMol;
    long long* const gmsd = gh + 512;
    long long myMsd = 0;
    uint32_t const lane = threadIdx.x & 31u;
    // npad is a multiple of 32 and so is the grid's stride: every lane of a warp runs the same
    // iterations, so the warp-wide reduction below sees all 32 lanes
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < S.npad; g += gridDim.x * blockDim.x) {
        uint32_t const m = o.molOfSlot[g];
        bool const real = m != kNoColor;   // padding slots add nothing
        int32_t const ix = real ? slot_coord(S, g, 0) : 0, iy = real ? slot_coord(S, g, 1) : 0,
                      iz = real ? slot_coord(S, g, 2) : 0;
        long long const x = ix, y = iy, z = iz;
        // per-molecule sums: the lanes of a warp mostly hold monomers of one or two chains, so they
        // are summed over each run of equal molecule ids first (a segmented scan; run r starts at
        // the highest run head at or below the lane) and the run's last lane adds them, one atomic
        // per run and sum instead of one per monomer; integer sums are exact in any order
        uint32_t const mPrev = __shfl_up_sync(0xffffffffu, m, 1);
        unsigned const heads = __ballot_sync(0xffffffffu, lane == 0 || mPrev != m);
        uint32_t const runStart = 31u - __clz(heads & (0xffffffffu >> (31u - lane)));
        bool const runEnd = lane == 31u || ((heads >> (lane + 1u)) & 1u);
        long long sum[4] = {x, y, z, x * x + y * y + z * z};
#pragma unroll
        for (uint32_t off = 1; off < 32u; off <<= 1) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                long long const v = __shfl_up_sync(0xffffffffu, sum[c], off);
                if (lane >= runStart + off) sum[c] += v;
            }
        }
        if (real && runEnd)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                atomicAdd(reinterpret_cast<unsigned long long*>(mom + 4ull * m + c), (unsigned long long)sum[c]);
        if (!real) continue;
        long long const dx = x - o.rx[g], dy = y - o.ry[g], dz = z - o.rz[g];
        myMsd += dx * dx + dy * dy + dz * dz;
        uint32_t const nn = S.nnb[g];
        if (S.codeMode == kCodeNone) {
            for (uint32_t k = 0; k < nn; ++k) {
                uint32_t const j = S.nbr[(size_t)k * S.npad + g];
                atomicAdd(&hist[bond_index(S.x[j] - ix, S.y[j] - iy, S.z[j] - iz)], 1u);
            }
        } else {
            // field k of the slot's bond-code word is the bond index of (neighbour k - monomer), in
            // the order of the neighbour list
            unsigned long long const code = S.codeMode == kCode32 ? (unsigned long long)*rec_code<uint32_t>(S.rec, g)
                                                                  : *rec_code<unsigned long long>(S.rec, g);
            for (uint32_t k = 0; k < nn; ++k) atomicAdd(&hist[uint32_t(code >> (9u * k)) & 511u], 1u);
        }
    }
    for (int sh = 16; sh > 0; sh >>= 1) myMsd += __shfl_down_sync(0xffffffffu, myMsd, sh);
    if ((threadIdx.x & 31u) == 0 && myMsd) atomicAdd(reinterpret_cast<unsigned long long*>(&msd), (unsigned long long)myMsd);
    // end-to-end vectors, one thread per molecule
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < o.nMol; m += gridDim.x * blockDim.x) {
        uint32_t const a = o.ends[2 * m], b = o.ends[2 * m + 1];
        long long const dx = (long long)slot_coord(S, b, 0) - slot_coord(S, a, 0);
        long long const dy = (long long)slot_coord(S, b, 1) - slot_coord(S, a, 1);
        long long const dz = (long long)slot_coord(S, b, 2) - slot_coord(S, a, 2);
        ree[m] = dx * dx + dy * dy + dz * dz;
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < 512; b += blockDim.x)
        if (hist[b]) atomicAdd(reinterpret_cast<unsigned long long*>(gh + b), (unsigned long long)hist[b]);
    if (threadIdx.x == 0 && msd) atomicAdd(reinterpret_cast<unsigned long long*>(gmsd), (unsigned long long)msd);
}

cudaError_t launch_observables(SysDev const* dSys, ObsDev const& o, long long* dOut, uint32_t npad, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(dOut, 0, sizeof(long long) * obs_words(o.nMol), s);
    if (e != cudaSuccess) return e;
    uint32_t const grid = (npad + 255) / 256 < 1184 ? (npad + 255) / 256 : 1184;
    k_observables<<<grid ? grid : 1, 256, 0, s>>>(dSys, o, dOut);
    return cudaGetLastError();
}

}  // namespace bfm
