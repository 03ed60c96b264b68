// sm_100a kernels of the BFM sweep.
//
// One sub-step of the reference (src/pscbfm/CRITICAL.cu:501-573) is: draw a colour c and a
// 32-bit seed, run the check kernel over colour group c (CRITICAL.cu:298-374), run the
// perform-and-apply kernel (CRITICAL.cu:376-411), clear the temporary lattice (:561-573).
//
// Two kernel families implement it:
//  * grid phase (k_check, k_perform): one launch per phase over a tile list that may span many
//    systems (one system for the drop-in path, a whole ensemble for the batched path). The
//    temporary lattice is double-buffered; the perform launch of sub-step t also zeroes the
//    words marked by sub-step t-1 (tmark), so no memset of the whole lattice is ever needed.
//  * resident (k_resident): one CTA owns one small system (box <= 64^3) for a whole chunk of
//    MCS. Occupancy and both temporary lattices live in shared memory; __syncthreads is the
//    barrier between check and perform; tentative flags stay in registers.
// Both produce exactly the reference's trajectory: the check reads only the pre-sub-step
// lattice and positions, the perform reads only the temporary lattice, and every write of the
// perform phase is a disjoint move (no two accepted movers touch the same cell).

#include <cuda_runtime.h>

#include <algorithm>

#include <cstdint>

#include "bfm_device.cuh"
#include "bfm_kernels.hpp"

namespace bfm {

namespace {

__device__ __forceinline__ void dir_vec(uint32_t dir, int32_t& dx, int32_t& dy, int32_t& dz)
{
    int32_t const s = (dir & 1u) ? 1 : -1;
    uint32_t const a = dir >> 1;
    dx = a == 0 ? s : 0;
    dy = a == 1 ? s : 0;
    dz = a == 2 ? s : 0;
}

__device__ __forceinline__ void load_sys(SysDev& dst, SysDev const* src)
{
    static_assert(sizeof(SysDev) % 4 == 0, "SysDev is copied word by word");
    uint32_t const* s = reinterpret_cast<uint32_t const*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (uint32_t w = threadIdx.x; w < sizeof(SysDev) / 4; w += blockDim.x) d[w] = s[w];
}

}  // namespace

// ------------------------------------------------------------------------ grid phase: check

__global__ void __launch_bounds__(kGridBlock) k_check(SysDev const* __restrict__ sysv,
                                                      TileRef const* __restrict__ tiles, uint32_t tileSpan,
                                                      StepEntry const* __restrict__ steps)
{
    __shared__ SysDev S;
    __shared__ uint32_t tally;
    TileRef const tr = tiles ? tiles[blockIdx.x] : TileRef{0u, blockIdx.x * tileSpan};
    StepEntry const st = steps[tr.sys];
    if (st.color == kNoColor) return;
    load_sys(S, sysv + tr.sys);
    if (threadIdx.x == 0) tally = 0;
    __syncthreads();

    uint32_t const off = S.grp[2 * st.color], cnt = S.grp[2 * st.color + 1];
    unsigned long long* const tmpCur = S.tmp + (size_t)st.parity * S.nwords;
    uint32_t* const markCur = S.tmark + (size_t)st.parity * S.npad;
    unsigned long long const* const lat = S.lat;
    auto loadLat = [lat](uint32_t w) { return __ldg(lat + w); };

    uint32_t const end = min(tr.start + tileSpan, ((cnt + 31u) & ~31u));
    for (uint32_t i = tr.start + threadIdx.x; i < end; i += blockDim.x) {
        bool const live = i < cnt;
        bool ok = false;
        if (live) {
            uint32_t const g = off + i;
            int32_t const x0 = __ldg(S.x + g), y0 = __ldg(S.y + g), z0 = __ldg(S.z + g);
            uint32_t const dir = move_dir(i, st.seed);
            int32_t dx, dy, dz;
            dir_vec(dir, dx, dy, dz);
            int32_t const x1 = x0 + dx, y1 = y0 + dy, z1 = z0 + dz;
            uint32_t const nn = __ldg(S.nnb + g);
            uint32_t const ca = (dir >> 1) == 0 ? uint32_t(x0) : ((dir >> 1) == 1 ? uint32_t(y0) : uint32_t(z0));
            ok = !wall_blocks(S.walls, ca, dir, S.lim);
            for (uint32_t k = 0; k < nn; ++k) {
                uint32_t const j = __ldg(S.nbr + (size_t)k * S.npad + g);
                uint32_t const idx = bond_index(__ldg(S.x + j) - x1, __ldg(S.y + j) - y1, __ldg(S.z + j) - z1);
                if (forbidden(S.forbid, idx)) ok = false;
            }
            if (ok) ok = !front_occupied(loadLat, S.brickTab, S.nb, S.mask, x0, y0, z0, dir);
            uint8_t f = 0;
            uint32_t mark = kNoMark;
            if (ok) {
                uint32_t const w = brick_word(S.brickTab, S.nb, uint32_t(x1) & S.mask[0], uint32_t(y1) & S.mask[1],
                                              uint32_t(z1) & S.mask[2]);
                uint32_t const b = brick_bit(uint32_t(x1), uint32_t(y1), uint32_t(z1));
                atomicOr(tmpCur + w, 1ull << b);
                f = (uint8_t)((dir << 2) | 1u);
                mark = (w << 6) | b;
            }
            S.flags[g] = f;
            markCur[g] = mark;
        }
        tally_warp(ok, &tally);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        tally_flush(tally, S.stats, 1);
        if (tr.start == 0) tally_flush(cnt, S.stats, 0);
    }
}

// ------------------------------------------------------------------------ grid phase: perform

__global__ void __launch_bounds__(kGridBlock) k_perform(SysDev const* __restrict__ sysv,
                                                        TileRef const* __restrict__ tiles, uint32_t tileSpan,
                                                        StepEntry const* __restrict__ steps, StepEntry* next)
{
    __shared__ SysDev S;
    __shared__ uint32_t tally;
    TileRef const tr = tiles ? tiles[blockIdx.x] : TileRef{0u, blockIdx.x * tileSpan};
    StepEntry const st = steps[tr.sys];
    if (st.color == kNoColor && st.prevColor == kNoColor) return;
    load_sys(S, sysv + tr.sys);
    if (threadIdx.x == 0) tally = 0;
    __syncthreads();
    // one system in a captured graph: hand the next launch its entry (write_next_step)
    if (next != nullptr && blockIdx.x == 0 && threadIdx.x == 0) write_next_step(S.gen, *S.gen, S.grp, next);

    // scrub the marks of the previous sub-step of this system (other parity)
    if (st.prevColor != kNoColor) {
        uint32_t const poff = S.grp[2 * st.prevColor], pcnt = S.grp[2 * st.prevColor + 1];
        uint32_t const pend = min(tr.start + tileSpan, pcnt);
        unsigned long long* const tmpPrev = S.tmp + (size_t)(st.parity ^ 1u) * S.nwords;
        uint32_t const* const markPrev = S.tmark + (size_t)(st.parity ^ 1u) * S.npad;
        for (uint32_t i = tr.start + threadIdx.x; i < pend; i += blockDim.x) {
            uint32_t const m = markPrev[poff + i];
            // every set bit of this buffer belongs to a mover of the previous sub-step, so
            // zeroing the whole word clears only bits that are due to be cleared
            if (m != kNoMark) tmpPrev[m >> 6] = 0ull;
        }
    }
    if (st.color == kNoColor) return;

    uint32_t const off = S.grp[2 * st.color], cnt = S.grp[2 * st.color + 1];
    unsigned long long const* const tmpCur = S.tmp + (size_t)st.parity * S.nwords;
    auto loadTmp = [tmpCur](uint32_t w) { return __ldg(tmpCur + w); };
    uint32_t const end = min(tr.start + tileSpan, ((cnt + 31u) & ~31u));
    for (uint32_t i = tr.start + threadIdx.x; i < end; i += blockDim.x) {
        bool moved = false;
        if (i < cnt) {
            uint32_t const g = off + i;
            uint8_t const f = S.flags[g];
            if (f & 1u) {
                uint32_t const dir = (f >> 2) & 7u;
                int32_t const x0 = S.x[g], y0 = S.y[g], z0 = S.z[g];
                if (!front_occupied(loadTmp, S.brickTab, S.nb, S.mask, x0, y0, z0, dir)) {
                    int32_t dx, dy, dz;
                    dir_vec(dir, dx, dy, dz);
                    int32_t const x1 = x0 + dx, y1 = y0 + dy, z1 = z0 + dz;
                    uint32_t const w0 = brick_word(S.brickTab, S.nb, uint32_t(x0) & S.mask[0],
                                                   uint32_t(y0) & S.mask[1], uint32_t(z0) & S.mask[2]);
                    uint32_t const w1 = brick_word(S.brickTab, S.nb, uint32_t(x1) & S.mask[0],
                                                   uint32_t(y1) & S.mask[1], uint32_t(z1) & S.mask[2]);
                    unsigned long long const b0 = 1ull << brick_bit(uint32_t(x0), uint32_t(y0), uint32_t(z0));
                    unsigned long long const b1 = 1ull << brick_bit(uint32_t(x1), uint32_t(y1), uint32_t(z1));
                    if (w0 == w1) {
                        atomicXor(S.lat + w0, b0 | b1);
                    } else {
                        atomicXor(S.lat + w0, b0);
                        atomicXor(S.lat + w1, b1);
                    }
                    uint32_t const a = dir >> 1;
                    if (a == 0) S.x[g] = x1;
                    else if (a == 1) S.y[g] = y1;
                    else S.z[g] = z1;
                    moved = true;
                }
            }
        }
        tally_warp(moved, &tally);
    }
    __syncthreads();
    if (threadIdx.x == 0) tally_flush(tally, S.stats, 2);
}

// ------------------------------------------------------------------------ resident (1 CTA / system)

template <int K>
__global__ void __launch_bounds__(kResidentBlock, 1) k_resident(SysDev const* __restrict__ sysv,
                                                                 uint32_t const* __restrict__ sysList,
                                                                 StepEntry const* __restrict__ steps, uint32_t nSys,
                                                                 uint32_t nSteps)
{
    __shared__ SysDev S;
    extern __shared__ unsigned long long smem[];
    uint32_t const sysId = sysList[blockIdx.x];
    load_sys(S, sysv + sysId);
    __syncthreads();

    uint32_t const nw = S.nwords;
    unsigned long long* const lat = smem;
    unsigned long long* const tmpA = smem + nw;
    unsigned long long* const tmpB = smem + 2 * nw;
    uint32_t* const tab = reinterpret_cast<uint32_t*>(smem + 3 * nw);
    uint32_t const ntab = S.nb[0] + S.nb[1] + S.nb[2];
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        lat[w] = S.lat[w];
        tmpA[w] = 0ull;
        tmpB[w] = 0ull;
    }
    for (uint32_t w = threadIdx.x; w < ntab; w += blockDim.x) tab[w] = S.brickTab[w];
    __syncthreads();

    auto loadLat = [lat](uint32_t w) { return lat[w]; };
    int32_t* const X = S.x;
    int32_t* const Y = S.y;
    int32_t* const Z = S.z;
    uint32_t nTent = 0, nAcc = 0;
    unsigned long long nAtt = 0;

    for (uint32_t t = 0; t < nSteps; ++t) {
        StepEntry const st = steps[(size_t)t * nSys + sysId];
        if (st.color == kNoColor) continue;
        unsigned long long* const cur = (t & 1u) ? tmpB : tmpA;
        unsigned long long* const other = (t & 1u) ? tmpA : tmpB;
        uint32_t const off = S.grp[2 * st.color], cnt = S.grp[2 * st.color + 1];
        nAtt += cnt;
        // check: clear the buffer of the next sub-step, mark tentative targets in `cur`
        for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) other[w] = 0ull;
        uint8_t fl[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            uint32_t const i = threadIdx.x + (uint32_t)k * blockDim.x;
            fl[k] = 0;
            if (i < cnt) {
                uint32_t const g = off + i;
                int32_t const x0 = X[g], y0 = Y[g], z0 = Z[g];
                uint32_t const dir = move_dir(i, st.seed);
                int32_t dx, dy, dz;
                dir_vec(dir, dx, dy, dz);
                int32_t const x1 = x0 + dx, y1 = y0 + dy, z1 = z0 + dz;
                uint32_t const nn = S.nnb[g];
                uint32_t const ca = (dir >> 1) == 0 ? uint32_t(x0) : ((dir >> 1) == 1 ? uint32_t(y0) : uint32_t(z0));
                bool ok = !wall_blocks(S.walls, ca, dir, S.lim);
                for (uint32_t q = 0; q < nn; ++q) {
                    uint32_t const j = S.nbr[(size_t)q * S.npad + g];
                    if (forbidden(S.forbid, bond_index(X[j] - x1, Y[j] - y1, Z[j] - z1))) ok = false;
                }
                if (ok && !front_occupied(loadLat, tab, S.nb, S.mask, x0, y0, z0, dir)) {
                    uint32_t const w = brick_word(tab, S.nb, uint32_t(x1) & S.mask[0], uint32_t(y1) & S.mask[1],
                                                  uint32_t(z1) & S.mask[2]);
                    atomicOr(cur + w, 1ull << brick_bit(uint32_t(x1), uint32_t(y1), uint32_t(z1)));
                    fl[k] = (uint8_t)((dir << 2) | 1u);
                    ++nTent;
                }
            }
        }
        __syncthreads();
        // perform: re-check against the tentative targets, apply
        auto loadCur = [cur](uint32_t w) { return cur[w]; };
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!(fl[k] & 1u)) continue;
            uint32_t const i = threadIdx.x + (uint32_t)k * blockDim.x;
            uint32_t const g = off + i;
            uint32_t const dir = (fl[k] >> 2) & 7u;
            int32_t const x0 = X[g], y0 = Y[g], z0 = Z[g];
            if (front_occupied(loadCur, tab, S.nb, S.mask, x0, y0, z0, dir)) continue;
            int32_t dx, dy, dz;
            dir_vec(dir, dx, dy, dz);
            int32_t const x1 = x0 + dx, y1 = y0 + dy, z1 = z0 + dz;
            uint32_t const w0 = brick_word(tab, S.nb, uint32_t(x0) & S.mask[0], uint32_t(y0) & S.mask[1],
                                           uint32_t(z0) & S.mask[2]);
            uint32_t const w1 = brick_word(tab, S.nb, uint32_t(x1) & S.mask[0], uint32_t(y1) & S.mask[1],
                                           uint32_t(z1) & S.mask[2]);
            unsigned long long const b0 = 1ull << brick_bit(uint32_t(x0), uint32_t(y0), uint32_t(z0));
            unsigned long long const b1 = 1ull << brick_bit(uint32_t(x1), uint32_t(y1), uint32_t(z1));
            if (w0 == w1) {
                atomicXor(lat + w0, b0 | b1);
            } else {
                atomicXor(lat + w0, b0);
                atomicXor(lat + w1, b1);
            }
            uint32_t const a = dir >> 1;
            if (a == 0) X[g] = x1;
            else if (a == 1) Y[g] = y1;
            else Z[g] = z1;
            ++nAcc;
        }
        __syncthreads();
    }
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) S.lat[w] = lat[w];
    // per-CTA statistics
    uint32_t tsum = __reduce_add_sync(0xffffffffu, nTent);
    uint32_t asum = __reduce_add_sync(0xffffffffu, nAcc);
    if ((threadIdx.x & 31u) == 0) {
        tally_flush(tsum, S.stats, 1);
        tally_flush(asum, S.stats, 2);
    }
    if (threadIdx.x == 0 && nAtt) atomicAdd(S.stats + (blockIdx.x % kStatSlots), nAtt);
}

// ------------------------------------------------------------------------ lattice build

__global__ void k_build_lattice(SysDev const* __restrict__ sysv, uint32_t n)
{
    SysDev const& S = sysv[0];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        int32_t const x = S.x[g], y = S.y[g], z = S.z[g];
        if (x == kPadCoord) continue;
        uint32_t const w = brick_word(S.brickTab, S.nb, uint32_t(x) & S.mask[0], uint32_t(y) & S.mask[1],
                                      uint32_t(z) & S.mask[2]);
        atomicOr(S.lat + w, 1ull << brick_bit(uint32_t(x), uint32_t(y), uint32_t(z)));
    }
}

// ------------------------------------------------------------------------ position read-back

// Positions in the caller's monomer order, x y z interleaved: out[3 i + a] is coordinate a of the
// monomer in sorted slot slotOf[i]. One copy of out then gives the caller's array. With bond codes
// (rec != nullptr) x, y, z hold image offsets and the lattice address the rest (slot_coord).
__global__ void k_gather_positions(int32_t const* __restrict__ x, int32_t const* __restrict__ y,
                                   int32_t const* __restrict__ z, uint32_t const* __restrict__ rec, uint32_t recWords,
                                   uint32_t m0, uint32_t m1, uint32_t m2, uint32_t const* __restrict__ slotOf,
                                   uint32_t n, int32_t* __restrict__ out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t const g = slotOf[i];
        int32_t cx = x[g], cy = y[g], cz = z[g];
        if (rec != nullptr) {
            uint32_t const p = rec[(size_t)g * recWords];
            cx += int32_t(axis_coord(p, m0));
            cy += int32_t(axis_coord(p, m1));
            cz += int32_t(axis_coord(p, m2));
        }
        out[3ull * i] = cx;
        out[3ull * i + 1] = cy;
        out[3ull * i + 2] = cz;
    }
}

// Unfolded positions of every slot of a bond-code system in slot order (the MSD reference of the
// observables); padding slots keep kPadCoord.
__global__ void k_unfold_positions(SysDev const* __restrict__ sysv, int32_t* __restrict__ ox,
                                   int32_t* __restrict__ oy, int32_t* __restrict__ oz)
{
    SysDev const& S = sysv[0];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < S.npad; g += gridDim.x * blockDim.x) {
        ox[g] = slot_coord(S, g, 0);
        oy[g] = slot_coord(S, g, 1);
        oz[g] = slot_coord(S, g, 2);
    }
}

// One warp: each counter's slots summed with a warp reduction, written to host memory. The host
// reads them only after an event behind this kernel has completed, so no fence is needed here.
__global__ void k_publish_stats(unsigned long long const* __restrict__ stats, unsigned long long* __restrict__ out)
{
    uint32_t const lane = threadIdx.x;
    for (uint32_t c = 0; c < 3; ++c) {
        unsigned long long v = 0;
        for (uint32_t k = lane; k < kStatSlots; k += 32) v += stats[c * kStatSlots + k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) out[c] = v;
    }
}

__global__ void k_snapshot_stats(unsigned long long const* __restrict__ stats, unsigned long long* ring,
                                 unsigned long long* seq)
{
    snapshot_stats(stats, ring, seq);
}

// One thread: snapshot slot (4 words) into host memory (mapped), the sequence number included.
__global__ void k_publish_snap(unsigned long long const* __restrict__ slot, unsigned long long* __restrict__ out)
{
    if (threadIdx.x < 4) out[threadIdx.x] = slot[threadIdx.x];
}

// ------------------------------------------------------------------------ launchers

cudaError_t launch_check(SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles, uint32_t tileSpan,
                         StepEntry const* dSteps, cudaStream_t s)
{
    if (nTiles == 0) return cudaSuccess;
    k_check<<<nTiles, kGridBlock, 0, s>>>(dSys, dTiles, tileSpan, dSteps);
    return cudaGetLastError();
}

cudaError_t launch_perform(SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles, uint32_t tileSpan,
                           StepEntry const* dSteps, cudaStream_t s, StepEntry* next)
{
    if (nTiles == 0) return cudaSuccess;
    k_perform<<<nTiles, kGridBlock, 0, s>>>(dSys, dTiles, tileSpan, dSteps, next);
    return cudaGetLastError();
}

size_t resident_smem_bytes(uint32_t nwords, uint32_t ntab)
{
    return (size_t)nwords * 3 * sizeof(unsigned long long) + (size_t)ntab * sizeof(uint32_t);
}

template <int K>
static cudaError_t launch_resident_k(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, StepEntry const* dSteps,
                                     uint32_t nSys, uint32_t nSteps, size_t smem, cudaStream_t s)
{
    // the attribute is per function and per device context; raise it to what this launch needs
    static thread_local size_t attrSet[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    size_t& have = attrSet[dev & 63];
    if (smem > have) {
        e = cudaFuncSetAttribute(k_resident<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        have = smem;
    }
    k_resident<K><<<nCta, kResidentBlock, smem, s>>>(dSys, dList, dSteps, nSys, nSteps);
    return cudaGetLastError();
}

cudaError_t launch_resident(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, uint32_t perThread,
                            StepEntry const* dSteps, uint32_t nSys, uint32_t nSteps, size_t smem, cudaStream_t s)
{
    if (nCta == 0 || nSteps == 0) return cudaSuccess;
    if (smem > kResidentMaxSmem) return cudaErrorInvalidValue;
    switch (perThread) {
    case 1: return launch_resident_k<1>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 2: return launch_resident_k<2>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 4: return launch_resident_k<4>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 8: return launch_resident_k<8>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 16: return launch_resident_k<16>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gather_positions(SysDev const& h, uint32_t const* slotOf, uint32_t n, int32_t* out,
                                    cudaStream_t s)
{
    uint32_t const block = 256;
    uint32_t const grid = std::min((n + block - 1) / block, 148u * 8u);
    if (grid == 0) return cudaSuccess;
    bool const codes = h.codeMode != kCodeNone;
    k_gather_positions<<<grid, block, 0, s>>>(h.x, h.y, h.z, codes ? h.rec : nullptr, rec_words(h.codeMode),
                                              h.amask[0], h.amask[1], h.amask[2], slotOf, n, out);
    return cudaGetLastError();
}

cudaError_t launch_unfold_positions(SysDev const* dSys, uint32_t npad, int32_t* ox, int32_t* oy, int32_t* oz,
                                    cudaStream_t s)
{
    uint32_t const block = 256;
    uint32_t const grid = std::min((npad + block - 1) / block, 148u * 8u);
    if (grid == 0) return cudaSuccess;
    k_unfold_positions<<<grid, block, 0, s>>>(dSys, ox, oy, oz);
    return cudaGetLastError();
}

cudaError_t launch_publish_stats(unsigned long long const* stats, unsigned long long* out, cudaStream_t s)
{
    k_publish_stats<<<1, 32, 0, s>>>(stats, out);
    return cudaGetLastError();
}

cudaError_t launch_snapshot_stats(unsigned long long const* stats, unsigned long long* ring, unsigned long long* seq,
                                  cudaStream_t s)
{
    k_snapshot_stats<<<1, 32, 0, s>>>(stats, ring, seq);
    return cudaGetLastError();
}

cudaError_t launch_publish_snap(unsigned long long const* slot, unsigned long long* out, cudaStream_t s)
{
    k_publish_snap<<<1, 32, 0, s>>>(slot, out);
    return cudaGetLastError();
}

cudaError_t launch_build_lattice(SysDev const* dSys, uint32_t npad, cudaStream_t s)
{
    uint32_t const block = 256;
    uint32_t const grid = (npad + block - 1) / block;
    if (grid == 0) return cudaSuccess;
    k_build_lattice<<<grid, block, 0, s>>>(dSys, npad);
    return cudaGetLastError();
}

}  // namespace bfm
