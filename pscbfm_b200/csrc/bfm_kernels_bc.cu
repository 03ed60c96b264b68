// Bond-code kernels of the BFM sweep (sm_100a).
//
// The same sub-step as the gather kernels (check: CRITICAL.cu:298-374, perform + apply:
// CRITICAL.cu:376-411, clear: :561-573), on a different state: each monomer keeps the lattice
// address of its corner (pk: brick word << 6 | bit; moves and front planes are adds confined to one
// axis's address bits) and a bond-code word whose 9-bit fields are the reference's bond-table
// indices of its bonds, so the check needs no neighbour positions. When a monomer moves by d, its
// own fields change by -d and the reverse field of every neighbour by +d; the reverse field's old
// value is the negation (mod 8) of the monomer's own field, so the update needs no extra load.
//
// Grid phase (k_check_bc, k_perform_bc): the check lists its tentative movers per tile, with the
// address of the temporary-lattice cell each one marked (mover lists, double-buffered by sub-step
// parity); the perform walks only those lists, and the perform of sub-step t also zeroes the words
// listed at t-1. Every independent load of a pass is issued before any dependent one; a single-system
// launch takes the descriptor as a grid-constant parameter.
//
// Persistent (k_sweep_bc): the same bodies for a whole run of sub-steps in one launch: a grid of
// at most 16 CTAs as one thread-block cluster with hardware barriers between the phases, a larger
// one as a cooperative launch with time-bounded grid barriers.
//
// Resident (k_resident_bc): one CTA owns a small system for a chunk of sub-steps; lattice, one
// temporary lattice, pk and bond codes in shared memory; the check appends tentative movers to a
// shared list (warp ballot + one atomic per warp), so the perform runs with full warps.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "bfm_device.cuh"
#include "bfm_kernels.hpp"

namespace bfm {

namespace {


__device__ __forceinline__ void copy_desc(SysDev& dst, SysDev const* src)
{
    static_assert(sizeof(SysDev) % 4 == 0, "SysDev is copied word by word");
    uint32_t const* s = reinterpret_cast<uint32_t const*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (uint32_t w = threadIdx.x; w < sizeof(SysDev) / 4; w += blockDim.x) d[w] = s[w];
}

// True if every bond of the code word stays allowed after the move along dir: the AND of the move
// table's entries over all fields (an unused field is index 0, whose entry allows every move).
template <typename W, bool kSharedTables>
__device__ __forceinline__ bool bonds_ok(W code, uint32_t dir, uint8_t const* ok)
{
    uint32_t m = 0xFFu;
#pragma unroll
    for (uint32_t k = 0; k < CodeWord<W>::kSlots; ++k) {
        uint32_t const idx = uint32_t(code >> (9u * k)) & 511u;
        m &= kSharedTables ? ok[idx] : __ldg(ok + idx);
    }
    return (m >> dir) & 1u;
}

// Loads of state the sweep changes (packed coordinates, codes, flags, lattices): through the
// read-only data path where one launch only reads them (kNc), plain loads in the persistent
// kernel, where other CTAs wrote them earlier in the same launch (the read-only path is not
// coherent with those writes).
template <bool kNc, typename T>
__device__ __forceinline__ T ldm(T const* p)
{
    if constexpr (kNc) return __ldg(p);
    else return *p;
}

// Mover lists: the check of sub-step t appends each tentative mover of tile k (kBcTileSpan
// in-colour indices) to segment k of list[parity] (entry: slot g in bits 0-26, direction in
// 27-29), the lattice address of its target (the temporary-lattice cell it marked) to the same
// place of word[parity], and stores the segment's length in count[parity][k]. The perform of
// sub-step t walks only the listed movers, and zeroes the words of the targets listed at t-1
// (nobody reads tmp[parity^1] during sub-step t, and the check of t+1, which marks it again,
// comes after).
constexpr uint32_t kEntSlotMask = (1u << 27) - 1u;
// Tentative movers a lane of the grid perform takes per pass over its tile's list: 32 x kPerfQ
// entries, loaded together with the list's length (about a sixth of a dense tile's 512 monomers
// move tentatively, so one pass covers a tile of a dense system; longer lists take more passes).
constexpr int kPerfQ = 4;

// ---------------------------------------------------------------------------------- check

template <typename W, int MPT, bool kNc = true>
__device__ __forceinline__ void check_body(SysDev const& S, uint32_t const* dtab, StepEntry const& st, uint32_t start,
                                           uint32_t* segCount, uint2* stage)
{
    uint32_t const B = blockDim.x, tid = threadIdx.x;
    using RV = typename SlotRec<W>::V;
    RV const* const REC = reinterpret_cast<RV const*>(S.rec);
    uint32_t const tile = start / kBcTileSpan;
    unsigned long long* const tcur = S.tmp + (size_t)st.parity * S.nwords;
    size_t const seg = (size_t)st.parity * S.listStride + (size_t)tile * kBcTileSpan;
    uint32_t* const lcur = S.mlist + seg;
    uint32_t* const wcur = S.mword + seg;

    // stage 1: every independent load of the pass; they stay in flight across the barrier that
    // publishes the caller's shared writes (the direction table, the segment count)
    uint32_t pk[MPT];
    W code[MPT];
#pragma unroll
    for (int q = 0; q < MPT; ++q) {
        uint32_t const i = start + tid + (uint32_t)q * B;
        RV const r = i < st.cnt ? ldm<kNc>(REC + st.off + i) : RV{};
        pk[q] = r.x;
        code[q] = rec_code_of(r);
    }
    __syncthreads();
    // stage 2: direction, walls, bonds; the monomers that pass go to this warp's part of the
    // stage (address, slot | direction << 27), packed, so that the front-plane and occupancy work
    // below runs on full warps of candidates only (about half the monomers fail here)
    uint32_t const lane = tid & 31u;
    uint32_t const lanesBelow = (1u << lane) - 1u;
    uint2* const ws = stage + (tid >> 5) * (32u * MPT);
    uint32_t n = 0;
    bool const walled = S.walls != 0u;   // uniform: a periodic box skips the wall test's table reads
#pragma unroll
    for (int q = 0; q < MPT; ++q) {
        uint32_t const i = start + tid + (uint32_t)q * B;
        uint32_t const dir = move_dir(i, st.seed);
        bool free = true;
        if (walled) {
            uint2 const mw = make_uint2(dtab[dir * 4u], dtab[kDirHalf + dir * 4u + 3u]);   // Ma, wall
            free = (pk[q] & mw.x) != mw.y;
        }
        bool const ok = i < st.cnt && free && bonds_ok<W, false>(code[q], dir, S.moveOk);
        uint32_t const bal = __ballot_sync(0xffffffffu, ok);
        if (ok) ws[n + __popc(bal & lanesBelow)] = make_uint2(pk[q], (st.off + i) | (dir << 27));
        n += (uint32_t)__popc(bal);
    }
    __syncwarp();
    // stage 3: per candidate, the front plane from its address, the occupancy words, and for a
    // free plane the mark and the list entries (one shared-memory atomic per warp and pass)
    for (uint32_t b = 0; b < n; b += 32u) {
        bool const live = b + lane < n;
        uint2 const it = live ? ws[b + lane] : make_uint2(0u, 0u);
        uint32_t const dir = it.y >> 27;   // 0 for a dead lane: table reads stay in range
        DirParams const D = dir_params(dtab, dir);
        Plane pl;
        front_plane<false>(pl, S.planeTab, D, it.x, D.front, dir);
        uint32_t const to = addr_add(it.x, D.ma, D.step);
        unsigned long long hit = 0ull;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (live && ((pl.touch >> r) & 1u)) hit |= ldm<kNc>(S.lat + pl.w[r]) & pl.m[r];
        bool const go = live && hit == 0ull;
        uint32_t const bal = __ballot_sync(0xffffffffu, go);
        uint32_t base = 0;
        if (lane == 0 && bal) base = atomicAdd(segCount, (uint32_t)__popc(bal));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (go) {
            atomicOr(tcur + (to >> 6), 1ull << (to & 63u));
            uint32_t const slot = base + __popc(bal & lanesBelow);
            lcur[slot] = it.y;
            wcur[slot] = to;
        }
    }
}

// ---------------------------------------------------------------------------------- perform

// Image offsets (x, y, z with bond codes, see SysDev) of slot g after a move along axis a by s from
// lattice address p0 to p1 (ma: the axis's address bits): they change only when the move wraps the
// periodic axis, i.e. reaches coordinate 0 going up or leaves it going down; a walled axis never
// wraps. About one move in a lattice side along that axis writes here.
__device__ __forceinline__ void image_step(SysDev const& S, uint32_t g, uint32_t a, int32_t s, uint32_t p0,
                                           uint32_t p1, uint32_t ma)
{
    if (((s > 0 ? p1 : p0) & ma) == 0u)
        atomicAdd((a == 0 ? S.x : (a == 1 ? S.y : S.z)) + g, s * int32_t(S.mask[a] + 1u));
}

// Movers ent[q] (list entries: slot | direction << 27) with targets to[q], for the q with
// live[q]: re-test the front plane on the temporary lattice and apply the free moves. The plane
// and the old position follow from the target's address, so the monomer's own address is not
// loaded. Returns the moves applied.
template <typename W, int N, bool kNc>
__device__ __forceinline__ uint32_t perform_movers(SysDev const& S, uint32_t const* dtab,
                                                   unsigned long long const* tcur, uint32_t const (&ent)[N],
                                                   uint32_t const (&to)[N], bool const (&live)[N])
{
    using RV = typename SlotRec<W>::V;
    RV* const REC = reinterpret_cast<RV*>(S.rec);
    Plane pl[N];
    W code[N];
    uint32_t nbr[N][CodeWord<W>::kSlots];
#pragma unroll
    for (int q = 0; q < N; ++q) {
        uint32_t const g = live[q] ? ent[q] & kEntSlotMask : 0u;
        code[q] = live[q] ? *rec_code<W>(S.rec, g) : W(0);
#pragma unroll
        for (uint32_t k = 0; k < CodeWord<W>::kSlots; ++k)
            nbr[q][k] = (live[q] && k < S.maxc) ? __ldg(S.nbrr + (size_t)k * S.npad + g) : 0u;
    }
#pragma unroll
    for (int q = 0; q < N; ++q) {
        // a lane past its list's end may hold any stale word: direction 0 keeps its table reads in
        // range (the direction table has six entries, the plane table three axes)
        uint32_t const d = live[q] ? (ent[q] >> 27) & 7u : 0u;
        DirParams const D = dir_params(dtab, d);
        front_plane<false>(pl[q], S.planeTab, D, to[q], D.step, d);
    }
    unsigned long long hit[N];
#pragma unroll
    for (int q = 0; q < N; ++q) {
        hit[q] = 0ull;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (live[q] && ((pl[q].touch >> r) & 1u)) hit[q] |= ldm<kNc>(tcur + pl[q].w[r]) & pl[q].m[r];
    }
    uint32_t nAcc = 0;
#pragma unroll
    for (int q = 0; q < N; ++q) {
        if (!live[q] || hit[q] != 0ull) continue;
        ++nAcc;
        uint32_t const g = ent[q] & kEntSlotMask;
        uint32_t const dir = (ent[q] >> 27) & 7u;
        uint32_t const a = dir >> 1;
        int32_t const s = (dir & 1u) ? 1 : -1;
        uint2 const ms = *reinterpret_cast<uint2 const*>(dtab + dir * 4u);   // words 0, 1: Ma, step
        uint32_t const pk1 = to[q];
        uint32_t const pk0 = addr_add(pk1, ms.x, addr_back(ms.x, ms.y));
        uint32_t const w0 = pk0 >> 6, w1 = pk1 >> 6;
        if (w0 == w1) {
            atomicXor(S.lat + w0, (1ull << (pk0 & 63u)) | (1ull << (pk1 & 63u)));
        } else {
            atomicXor(S.lat + w0, 1ull << (pk0 & 63u));
            atomicXor(S.lat + w1, 1ull << (pk1 & 63u));
        }
        image_step(S, g, a, s, pk0, pk1, ms.x);
        W const own = code[q];
        REC[g] = make_rec(pk1, code_shift(own, a, -s));   // new address and code word in one store
        uint32_t const n = uint32_t(own >> CodeWord<W>::kCountShift) & 7u;
#pragma unroll
        for (uint32_t k = 0; k < CodeWord<W>::kSlots; ++k) {
            if (k < n) {
                uint32_t const nb = nbr[q][k];
                uint32_t const c = (0u - (uint32_t(own >> (9u * k + 3u * a)) & 7u)) & 7u;   // reverse field
                uint32_t const nc = uint32_t(int32_t(c) + s) & 7u;
                atomicXor(rec_code<W>(S.rec, nb & kSlotMask), W(c ^ nc) << (9u * (nb >> kSlotShift) + 3u * a));
            }
        }
    }
    return nAcc;
}

// Entries e, e + B, ... (MPT of them, those below total) of the concatenated mover lists of nT
// tiles (pre: the lists' starting offsets, lbase / tbase: the first tile's segment of the entries
// and of the target addresses), through perform_movers. Returns the moves applied.
template <typename W, int MPT, bool kNc>
__device__ __forceinline__ uint32_t perform_chunk(SysDev const& S, uint32_t const* dtab,
                                                  unsigned long long const* tcur, uint32_t const* lbase,
                                                  uint32_t const* tbase, uint32_t const* pre, uint32_t nT,
                                                  uint32_t total, uint32_t e)
{
    uint32_t const B = blockDim.x;
    uint32_t ent[MPT], to[MPT];
    bool live[MPT];
#pragma unroll
    for (int q = 0; q < MPT; ++q) {
        uint32_t const eq = e + (uint32_t)q * B;
        uint32_t j = 0;
        while (j + 1 < nT && eq >= pre[j + 1]) ++j;
        live[q] = eq < total;
        uint32_t const li = j * kBcTileSpan + (eq - pre[j]);
        ent[q] = live[q] ? ldm<kNc>(lbase + li) : 0u;
        to[q] = live[q] ? ldm<kNc>(tbase + li) : 0u;
    }
    return perform_movers<W, MPT, kNc>(S, dtab, tcur, ent, to, live);
}

// The persistent sweep's perform. For tiles tile0 .. tile0+nT-1 (at most 16): zeroes the
// temporary-lattice words the previous sub-step's movers marked, then walks this sub-step's
// tentative movers as one dense range
// (no thread waits on a monomer that did not move). pre is 2 (nT+1) words of shared memory: the
// starting offsets of the current and of the previous lists. A tile's list counts only if the
// tile lies inside that sub-step's colour group (older lengths may remain in count[]). Every thread
// of the CTA calls this; st.color == kNoColor only scrubs.
template <typename W, int MPT, bool kNc = true>
__device__ __forceinline__ void perform_body(SysDev const& S, uint32_t const* dtab, StepEntry const& st,
                                             uint32_t tile0, uint32_t nT, uint32_t* tally, uint32_t* pre)
{
    uint32_t const B = blockDim.x, tid = threadIdx.x;
    unsigned long long const* const tcur = S.tmp + (size_t)st.parity * S.nwords;
    unsigned long long* const tprev = S.tmp + (size_t)(st.parity ^ 1u) * S.nwords;
    uint32_t const* const lbase = S.mlist + (size_t)st.parity * S.listStride + (size_t)tile0 * kBcTileSpan;
    uint32_t const* const tbase = S.mword + (size_t)st.parity * S.listStride + (size_t)tile0 * kBcTileSpan;
    uint32_t const* const wprev = S.mword + (size_t)(st.parity ^ 1u) * S.listStride + (size_t)tile0 * kBcTileSpan;
    uint32_t const* const cnt = S.mcount + (size_t)st.parity * S.countStride + tile0;
    uint32_t const* const cntPrev = S.mcount + (size_t)(st.parity ^ 1u) * S.countStride + tile0;
    uint32_t* const preP = pre + nT + 1;
    bool const active = st.color != kNoColor;
    // the list lengths, this sub-step's in lanes 0..nT-1 and the previous sub-step's in lanes
    // 16..16+nT-1, loaded by one warp before the barrier and scanned after it
    uint32_t const j = tid & 15u;
    uint32_t c = 0;
    if (tid < 32 && j < nT) {
        uint32_t const start = (tile0 + j) * kBcTileSpan;
        if (tid < 16) c = (active && start < st.cnt) ? ldm<kNc>(cnt + j) : 0u;
        else c = start < st.pcnt ? ldm<kNc>(cntPrev + j) : 0u;
    }
    __syncthreads();   // pre of an earlier call has been read; the caller's shared writes are visible
    if (tid < 32) {
#pragma unroll
        for (uint32_t o = 1; o < 16; o <<= 1) {
            uint32_t const v = __shfl_up_sync(0xffffffffu, c, o, 16);
            if (j >= o) c += v;
        }
        uint32_t* const dst = tid < 16 ? pre : preP;
        if (j < nT) dst[j + 1] = c;
        if (j == 0) dst[0] = 0u;
    }
    __syncthreads();
    // scrub of the previous sub-step: every set bit of tmp[parity^1] belongs to one of its
    // tentative movers, so zeroing a whole marked word only clears bits that are due. The first
    // words are loaded before the movers' chain starts and zeroed after it, so the two overlap.
    uint32_t const totalP = preP[nT];
    auto scrubWord = [&](uint32_t e) {
        uint32_t j = 0;
        while (j + 1 < nT && e >= preP[j + 1]) ++j;
        return ldm<kNc>(wprev + j * kBcTileSpan + (e - preP[j])) >> 6;
    };
    uint32_t const w0 = tid < totalP ? scrubWord(tid) : 0u;
    uint32_t const total = pre[nT];
    uint32_t nAcc = 0;
    for (uint32_t e0 = 0; e0 < total; e0 += B * MPT)
        nAcc += perform_chunk<W, MPT, kNc>(S, dtab, tcur, lbase, tbase, pre, nT, total, e0 + tid);
    if (tid < totalP) tprev[w0] = 0ull;
    for (uint32_t e = tid + B; e < totalP; e += B) tprev[scrubWord(e)] = 0ull;
    if (nAcc) atomicAdd(tally, nAcc);
}

// Grid-phase perform of one tile by a group of G warps (`sub` = this warp's index in the group):
// the group walks list segment `tile` of this sub-step (parity p: its tentative movers) and of the
// previous one (parity p ^ 1: it zeroes the temporary-lattice words those movers marked), warp
// `sub` taking entries sub * 32 + lane + 32 G q. Every load of the first pass is independent of the
// others: both list lengths and Q entries, target addresses and previous targets per lane come in
// one round trip, so no length scan or barrier precedes the movers' own loads; entries past a
// list's end lie inside the tile's segment and are ignored. The lengths are exact for every tile of
// the launch: a check CTA whose tile lies beyond its colour group stores a zero length. Longer lists
// take further passes. The warp's copy of the direction table (dtab) is written from d0, d1 (words
// lane and lane + 32, loaded by the caller) once those loads are out, so the table's round trip
// overlaps the lists'. Returns the moves this warp applied.
template <typename W, bool kNc, int Q>
__device__ __forceinline__ uint32_t perform_tile(SysDev const& S, uint32_t* dtab, uint32_t d0, uint32_t d1,
                                                 uint32_t p, uint32_t tile, bool doCur, bool doPrev, uint32_t sub,
                                                 uint32_t G, uint32_t& listLen)
{
    uint32_t const lane = threadIdx.x & 31u;
    size_t const seg = (size_t)tile * kBcTileSpan;
    uint32_t const* const lc = S.mlist + (size_t)p * S.listStride + seg;
    uint32_t const* const wc = S.mword + (size_t)p * S.listStride + seg;
    uint32_t const* const wp = S.mword + (size_t)(p ^ 1u) * S.listStride + seg;
    unsigned long long const* const tcur = S.tmp + (size_t)p * S.nwords;
    unsigned long long* const tprev = S.tmp + (size_t)(p ^ 1u) * S.nwords;
    uint32_t const cnt = doCur ? ldm<kNc>(S.mcount + (size_t)p * S.countStride + tile) : 0u;
    uint32_t const pcnt = doPrev ? ldm<kNc>(S.mcount + (size_t)(p ^ 1u) * S.countStride + tile) : 0u;
    listLen = cnt;
    uint32_t const first = sub * 32u + lane, stride = 32u * G;
    uint32_t ent[Q], to[Q], pw[Q];
    bool live[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        uint32_t const e = first + stride * (uint32_t)q;   // < 32 G Q <= kBcTileSpan
        ent[q] = doCur ? ldm<kNc>(lc + e) : 0u;
        to[q] = doCur ? ldm<kNc>(wc + e) : 0u;
        pw[q] = doPrev ? ldm<kNc>(wp + e) : 0u;
    }
    dtab[lane] = d0;
    if (lane + 32u < kDirTab) dtab[lane + 32u] = d1;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) live[q] = first + stride * (uint32_t)q < cnt;
    uint32_t nAcc = perform_movers<W, Q, kNc>(S, dtab, tcur, ent, to, live);
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (first + stride * (uint32_t)q < pcnt) tprev[pw[q] >> 6] = 0ull;
    uint32_t const pass = stride * (uint32_t)Q;
    for (uint32_t b = pass; b < cnt; b += pass) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const e = b + first + stride * (uint32_t)q;
            live[q] = e < cnt;
            ent[q] = live[q] ? ldm<kNc>(lc + e) : 0u;
            to[q] = live[q] ? ldm<kNc>(wc + e) : 0u;
        }
        nAcc += perform_movers<W, Q, kNc>(S, dtab, tcur, ent, to, live);
    }
    for (uint32_t b = pass; b < pcnt; b += pass) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const e = b + first + stride * (uint32_t)q;
            if (e < pcnt) tprev[ldm<kNc>(wp + e) >> 6] = 0ull;
        }
    }
    return nAcc;
}

}  // namespace

// ---------------------------------------------------------------------------------- kernels

// Grid-phase check: CTA b of B threads covers tile b (kBcTileSpan in-colour indices, kBcTileSpan / B
// per thread); a tile list (kMulti) gives each CTA its system and tile.
template <typename W, int B, bool kMulti, int kMinBlocks = 1>
__global__ void __launch_bounds__(B, kMinBlocks) k_check_bc(const __grid_constant__ SysDev S1,
                                                         SysDev const* __restrict__ sysv,
                                                         TileRef const* __restrict__ tiles,
                                                         StepEntry const* __restrict__ steps,
                                                         unsigned long long* snap)
{
    __shared__ SysDev Sm;
    __shared__ __align__(16) uint32_t dtab[kDirTab];
    constexpr int MPT = (int)kBcTileSpan / B;
    static_assert(B * MPT == (int)kBcTileSpan, "a CTA covers one list segment");
    // one system, snap != nullptr: the first warp of CTA 0 first takes the snapshot of the move
    // counters as the work before this launch left them (snapshot_stats). No CTA of the check adds to
    // the tentative count (the perform does) and CTA 0 adds the attempted count only after this, so
    // no other update of this launch can reach the counters before it.
    if (!kMulti && snap != nullptr && blockIdx.x == 0 && threadIdx.x < 32u)
        snapshot_stats(S1.stats, snap, snap + 4 * kSnapRing);
    uint32_t sys = 0, start = blockIdx.x * kBcTileSpan;
    // one system: the direction table's load goes out with the step entry's
    uint32_t dv = (!kMulti && threadIdx.x < kDirTab) ? S1.dirTab[threadIdx.x] : 0u;
    if (kMulti) {
        TileRef const tr = tiles[blockIdx.x];
        sys = tr.sys;
        start = tr.start;
    }
    StepEntry const st = steps[sys];
    if (st.color == kNoColor) return;
    if (start >= st.cnt) {
        // one system: the tile lies beyond this colour group; its list length becomes 0, so every
        // length the perform reads is this sub-step's (it does not read the step entry)
        if (!kMulti && threadIdx.x == 0) S1.mcount[(size_t)st.parity * S1.countStride + start / kBcTileSpan] = 0u;
        return;
    }
    if (kMulti) {
        copy_desc(Sm, sysv + sys);
        __syncthreads();
        if (threadIdx.x < kDirTab) dv = Sm.dirTab[threadIdx.x];
    }
    SysDev const& S = kMulti ? Sm : S1;
    __shared__ uint32_t segCount;
    __shared__ uint2 stage[kBcTileSpan];   // the warps' candidates (check_body)
    if (threadIdx.x < kDirTab) dtab[threadIdx.x] = dv;
    if (threadIdx.x == 0) segCount = 0;
    check_body<W, MPT>(S, dtab, st, start, &segCount, stage);   // publishes both with its first barrier
    __syncthreads();
    if (threadIdx.x == 0 && st.color != kNoColor) {
        // the list length; the perform that walks the list counts its entries as tentative moves
        S.mcount[(size_t)st.parity * S.countStride + start / kBcTileSpan] = segCount;
        if (start == 0) tally_flush(st.cnt, S.stats, 0);
    }
}

// Grid-phase perform: groups of G warps per tile of kBcTileSpan in-colour indices (perform_tile),
// PW warps per CTA (PW / G tiles); the groups of a CTA share nothing and never wait for each other.
// One system: `parity` and `scope` (kPerfCur: walk this sub-step's movers, kPerfPrev: scrub the
// previous sub-step's marks) come with the launch, so no load precedes the lists'; with parity ==
// kParityFromEntry they come from the step entry (a launch captured once and replayed on other
// entries). `next` != nullptr: the first warp of tile 0 also writes the following sub-step's entry
// there (write_next_step; the producer's state is loaded first, the entry stored after the warp's
// share of the tile). A tile list (kMulti): group b takes tile tiles[b] of system tiles[b].sys,
// whose step entry says what to do. nTiles: tiles of the launch (groups past it leave at once).
// Every warp of a group has 32 x max(4 / G, 1) list slots per pass.
template <typename W, bool kMulti, int PW, int G>
__global__ void __launch_bounds__(32 * PW) k_perform_bc(const __grid_constant__ SysDev S1, SysDev const* __restrict__ sysv,
                                                        TileRef const* __restrict__ tiles,
                                                        StepEntry const* __restrict__ steps, uint32_t parity,
                                                        uint32_t scope, StepEntry* next, uint32_t nTiles)
{
    static_assert(PW % G == 0, "whole groups per CTA");
    constexpr int Q = kPerfQ / G > 0 ? kPerfQ / G : 1;   // list slots per lane and pass
    __shared__ SysDev Sm[kMulti ? PW : 1];
    __shared__ __align__(16) uint32_t dtabs[PW][kDirTab];
    uint32_t const lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    uint32_t const wt = (blockIdx.x * PW + wid) / G;   // this group's tile (single) or tile-list entry
    uint32_t const sub = wid % G;
    if (wt >= nTiles) return;
    bool const writer = !kMulti && next != nullptr && wt == 0 && sub == 0 && lane == 0;
    StepGen gen{};
    if (writer) gen = *S1.gen;
    uint32_t p = parity, tile = wt, d0, d1;
    bool cur = (scope & kPerfCur) != 0u, prev = (scope & kPerfPrev) != 0u;
    if (!kMulti) {
        d0 = S1.dirTab[lane];
        d1 = lane + 32u < kDirTab ? S1.dirTab[lane + 32u] : 0u;
        if (parity == kParityFromEntry) {
            StepEntry const st = steps[0];
            uint32_t const start = tile * kBcTileSpan;
            p = st.parity;
            cur = st.color != kNoColor && start < st.cnt;
            prev = st.prevColor != kNoColor && start < st.pcnt;
        }
    } else {
        TileRef const tr = tiles[wt];
        SysDev& D = Sm[kMulti ? wid : 0];
        {   // the warp copies its system's descriptor
            static_assert(sizeof(SysDev) % 4 == 0, "SysDev is copied word by word");
            uint32_t const* src = reinterpret_cast<uint32_t const*>(sysv + tr.sys);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&D);
            for (uint32_t w = lane; w < sizeof(SysDev) / 4; w += 32u) dst[w] = src[w];
        }
        StepEntry const st = steps[tr.sys];
        p = st.parity;
        tile = tr.start / kBcTileSpan;
        cur = st.color != kNoColor && tr.start < st.cnt;
        prev = st.prevColor != kNoColor && tr.start < st.pcnt;
        __syncwarp();
        d0 = D.dirTab[lane];
        d1 = lane + 32u < kDirTab ? D.dirTab[lane + 32u] : 0u;
    }
    if (cur || prev) {
        SysDev const& S = kMulti ? Sm[kMulti ? wid : 0] : S1;
        uint32_t listLen = 0;
        uint32_t const nAcc = __reduce_add_sync(
            0xffffffffu,
            perform_tile<W, true, Q>(S, dtabs[wid], d0, d1, p, tile, cur, prev, sub, (uint32_t)G, listLen));
        uint32_t const stripe = (blockIdx.x * PW + wid) % kStatSlots;
        // the tile's list length (its tentative moves) is counted once, by the group's first warp
        if (lane == 0 && sub == 0 && listLen)
            atomicAdd(S.stats + kStatSlots + stripe, (unsigned long long)listLen);
        if (lane == 0 && nAcc) atomicAdd(S.stats + 2 * kStatSlots + stripe, (unsigned long long)nAcc);
    }
    if (writer) write_next_step(S1.gen, gen, S1.grp, next);
}

// ---------------------------------------------------------------------------------- persistent

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // a wait longer than 2 s is a fault

__device__ __forceinline__ unsigned int ld_acquire_gpu(unsigned int const* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_gpu_add(unsigned int* p, unsigned int v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// All CTAs of the cooperative grid meet; every write before the barrier is visible to every
// thread after it. After the CTA barrier, thread 0 adds the CTA's arrival to a count that only
// grows (a release add, which orders the whole CTA's earlier writes before it) and waits with
// acquire loads until the count reaches this barrier's target, gridDim.x above the previous one.
// Nothing is reset between barriers, and the signed difference keeps the comparison right
// across a wrap of the count. The wait is bounded by time and by a poll count; on every thread
// of the CTA it returns false if it ran out or another CTA's did (GridSync::fault): the kernel
// then leaves, and the host reports the fault.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned int& target, unsigned int* okSm)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ok = 1u;
        target += gridDim.x;
        red_release_gpu_add(&gs->count, 1u);
        if (int(ld_acquire_gpu(&gs->count) - target) < 0) {
            unsigned long long const t0 = global_ns();
            unsigned int polls = 0u;
            while (int(ld_acquire_gpu(&gs->count) - target) < 0) {
                // a time limit, and a poll count as a second bound that does not trust the timer
                if ((++polls & 255u) == 0u) {
                    if (ld_acquire_gpu(&gs->fault) != 0u) {
                        ok = 0u;
                        break;
                    }
                    if (global_ns() - t0 > kBarrierTimeoutNs || polls > (1u << 24)) {
                        if (atomicExch(&gs->fault, 1u) == 0u) gs->where = target / gridDim.x;
                        ok = 0u;
                        break;
                    }
                }
                __nanosleep(20);
            }
        }
        *okSm = ok;
    }
    __syncthreads();
    return *okSm != 0u;
}

// The whole grid as one thread-block cluster: the hardware cluster barrier, with release and
// acquire semantics at cluster scope, orders every thread's earlier global writes before any
// thread's later reads. Every CTA of the sweep reaches the same sequence of barriers.
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// One system, a whole run of sub-steps in one cooperative launch: per sub-step the check phase
// over every tile, a grid barrier, the perform phase and (between sub-steps) another barrier. CTA b
// takes tiles b, b + gridDim.x, ... of kGridBlock * MPT in-colour indices. Same bodies as
// k_check_bc / k_perform_bc, with plain loads of the state other CTAs change during the launch;
// the step entries are prefetched one sub-step ahead and the move counters flushed once.
template <typename W, int MPT, int kMinBlocks, bool kCluster, int B = (int)kGridBlock>
__global__ void __launch_bounds__(B, kMinBlocks)
    k_sweep_bc(const __grid_constant__ SysDev S, StepEntry const* __restrict__ steps, uint32_t nSteps,
               uint32_t nTiles, GridSync* gs)
{
    static_assert(B * MPT == (int)kBcTileSpan, "a tile is one list segment");
    __shared__ __align__(16) uint32_t dtab[kDirTab];
    __shared__ uint32_t tallyT, tallyA, okSm, segCount, pre[4];
    __shared__ uint2 stage[kBcTileSpan];   // the warps' candidates (check_body)
    if (ld_acquire_gpu(&gs->fault) != 0u) return;   // an earlier launch failed: the state is not usable
    if (threadIdx.x < kDirTab) dtab[threadIdx.x] = S.dirTab[threadIdx.x];
    if (threadIdx.x == 0) {
        tallyT = 0u;
        tallyA = 0u;
    }
    __syncthreads();
    constexpr uint32_t span = kBcTileSpan;
    unsigned int target = 0u;   // this CTA's count target of the next barrier
    unsigned long long att = 0ull;
    StepEntry next = steps[0];
    for (uint32_t t = 0; t < nSteps; ++t) {
        StepEntry const st = next;
        if (t + 1 < nSteps) next = steps[t + 1];
        bool const active = st.color != kNoColor;
        for (uint32_t k = blockIdx.x; k < nTiles; k += gridDim.x) {
            uint32_t const start = k * span;
            if (!active || start >= st.cnt) break;
            if (threadIdx.x == 0) segCount = 0u;   // published by check_body's first barrier
            check_body<W, MPT, false>(S, dtab, st, start, &segCount, stage);
            __syncthreads();
            if (threadIdx.x == 0) {
                S.mcount[(size_t)st.parity * S.countStride + k] = segCount;
                tallyT += segCount;
            }
        }
        if (active) att += st.cnt;
        if constexpr (kCluster) cluster_barrier();
        else if (!grid_barrier(gs, target, &okSm)) return;
        uint32_t const reach = max(active ? st.cnt : 0u, st.pcnt);   // movers now, marks of t-1
        for (uint32_t k = blockIdx.x; k < nTiles; k += gridDim.x) {
            if (k * span >= reach) break;
            perform_body<W, MPT, false>(S, dtab, st, k, 1u, &tallyA, pre);
        }
        if (t + 1 < nSteps) {
            if constexpr (kCluster) cluster_barrier();
            else if (!grid_barrier(gs, target, &okSm)) return;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        tally_flush(tallyT, S.stats, 1);
        tally_flush(tallyA, S.stats, 2);
        if (blockIdx.x == 0 && att) atomicAdd(S.stats, att);
    }
}

// ---------------------------------------------------------------------------------- resident

// The whole system in one CTA's shared memory for nSteps sub-steps: lattice, one temporary
// lattice per sub-step parity (the previous one cleared while the next check runs), packed
// coordinates, bond codes and the mover list; one CTA per system of sysList, entries of sub-step t
// at steps[t * nSys + system]. Two CTA barriers per sub-step (after the check, after the perform).
template <typename W, int K>
__global__ void __launch_bounds__(kResidentBlock, 1) k_resident_bc(SysDev const* __restrict__ sysv,
                                                                    uint32_t const* __restrict__ sysList,
                                                                    StepEntry const* __restrict__ steps,
                                                                    uint32_t nSys, uint32_t nSteps)
{
    __shared__ SysDev S;
    __shared__ uint32_t listCount[2];   // per sub-step parity
    extern __shared__ unsigned long long smem[];
    uint32_t const sysId = sysList[blockIdx.x];
    copy_desc(S, sysv + sysId);
    __syncthreads();
    uint32_t const nw = S.nwords, np = S.npad;
    uint32_t const B = blockDim.x, tid = threadIdx.x, lane = tid & 31u;
    unsigned long long* const ptab = smem;                  // 768 plane masks
    uint32_t* const dtab = reinterpret_cast<uint32_t*>(smem + 768);   // kDirTab words (16-byte aligned)
    unsigned long long* const lat = smem + 768 + kDirTab / 2;
    unsigned long long* const tmp = lat + nw;               // 2 x nw words (per sub-step parity)
    W* const code = reinterpret_cast<W*>(tmp + 2u * nw);
    uint32_t* const pk = reinterpret_cast<uint32_t*>(code + np);
    uint8_t* const mok = reinterpret_cast<uint8_t*>(pk + np);   // 512 move-table bytes
    uint32_t* const list = reinterpret_cast<uint32_t*>(mok + 512);
    for (uint32_t w = tid; w < 768; w += B) ptab[w] = S.planeTab[w];
    if (tid < kDirTab) dtab[tid] = S.dirTab[tid];
    for (uint32_t w = tid; w < 512; w += B) mok[w] = S.moveOk[w];
    for (uint32_t w = tid; w < nw; w += B) {
        lat[w] = S.lat[w];
        tmp[w] = 0ull;
        tmp[nw + w] = 0ull;
    }
    for (uint32_t g = tid; g < np; g += B) {
        code[g] = *rec_code<W>(S.rec, g);
        pk[g] = *rec_pk<W>(S.rec, g);
    }
    if (tid < 2) listCount[tid] = 0;
    uint32_t nTent = 0, nAcc = 0;
    unsigned long long nAtt = 0;
    StepEntry next = nSteps ? steps[sysId] : StepEntry{};
    __syncthreads();

    uint32_t par = 0;
    for (uint32_t t = 0; t < nSteps; ++t) {
        StepEntry const st = next;
        if (t + 1 < nSteps) next = steps[(size_t)(t + 1) * nSys + sysId];   // prefetch
        if (st.color == kNoColor) continue;
        nAtt += st.cnt;
        unsigned long long* const tmpCur = tmp + par * nw;
        // the previous sub-step's marks and list count: read by no thread after the barrier that
        // ended that sub-step, written by none before the barrier that ends this one
        for (uint32_t w = tid; w < nw; w += B) tmp[(par ^ 1u) * nw + w] = 0ull;
        if (tid == 0) listCount[par ^ 1u] = 0;
        // check: tentative movers -> tmp bit + shared list (one atomic per warp)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            uint32_t const i = tid + (uint32_t)k * B;
            bool go = false;
            uint32_t entry = 0;
            if (i < st.cnt) {
                uint32_t const g = st.off + i;
                uint32_t const dir = move_dir(i, st.seed);
                uint32_t const p = pk[g];
                DirParams const D = dir_params(dtab, dir);
                if ((p & D.ma) != D.wall && bonds_ok<W, true>(code[g], dir, mok)) {
                    Plane pl;
                    front_plane<true>(pl, ptab, D, p, D.front, dir);
                    unsigned long long hit = 0ull;
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                        if (pl.m[r]) hit |= lat[pl.w[r]] & pl.m[r];   // masks from shared memory
                    if (hit == 0ull) {
                        uint32_t const to = addr_add(p, D.ma, D.step);
                        atomicOr(tmpCur + (to >> 6), 1ull << (to & 63u));
                        go = true;
                        entry = g | (dir << kSlotShift);
                    }
                }
            }
            uint32_t const bal = __ballot_sync(0xffffffffu, go);
            if (bal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&listCount[par], (uint32_t)__popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (go) list[base + __popc(bal & ((1u << lane) - 1u))] = entry;
                nTent += lane == 0 ? (uint32_t)__popc(bal) : 0u;
            }
        }
        __syncthreads();
        // perform over the compact list
        uint32_t const nList = listCount[par];
        for (uint32_t e = tid; e < nList; e += B) {
            uint32_t const g = list[e] & kSlotMask, dir = list[e] >> kSlotShift;
            uint32_t const p = pk[g];
            // the neighbour references live in global memory: ask for them before the test, so
            // their latency overlaps it
            uint32_t nb[CodeWord<W>::kSlots];
#pragma unroll
            for (uint32_t q = 0; q < CodeWord<W>::kSlots; ++q)
                nb[q] = q < S.maxc ? __ldg(S.nbrr + (size_t)q * np + g) : 0u;
            Plane pl;
            DirParams const D = dir_params(dtab, dir);
            front_plane<true>(pl, ptab, D, p, D.front, dir);
            unsigned long long hit = 0ull;
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (pl.m[r]) hit |= tmpCur[pl.w[r]] & pl.m[r];
            if (hit != 0ull) continue;
            uint32_t const a = dir >> 1;
            int32_t const s = (dir & 1u) ? 1 : -1;
            uint32_t const p1 = addr_add(p, D.ma, D.step);
            uint32_t const w0 = p >> 6, w1 = p1 >> 6;
            if (w0 == w1) {
                atomicXor(lat + w0, (1ull << (p & 63u)) | (1ull << (p1 & 63u)));
            } else {
                atomicXor(lat + w0, 1ull << (p & 63u));
                atomicXor(lat + w1, 1ull << (p1 & 63u));
            }
            pk[g] = p1;
            image_step(S, g, a, s, p, p1, D.ma);
            W const own = code[g];
            code[g] = code_shift(own, a, -s);
            uint32_t const n = uint32_t(own >> CodeWord<W>::kCountShift) & 7u;
#pragma unroll
            for (uint32_t q = 0; q < CodeWord<W>::kSlots; ++q) {
                if (q < n) {
                    uint32_t const ent = nb[q];
                    uint32_t const c = (0u - (uint32_t(own >> (9u * q + 3u * a)) & 7u)) & 7u;
                    uint32_t const nc = uint32_t(int32_t(c) + s) & 7u;
                    atomicXor(code + (ent & kSlotMask), W(c ^ nc) << (9u * (ent >> kSlotShift) + 3u * a));
                }
            }
            ++nAcc;
        }
        __syncthreads();   // every perform is done: the lattice is settled for the next check
        par ^= 1u;
    }
    for (uint32_t w = tid; w < nw; w += B) S.lat[w] = lat[w];
    for (uint32_t g = tid; g < np; g += B) {
        *rec_code<W>(S.rec, g) = code[g];
        *rec_pk<W>(S.rec, g) = pk[g];
    }
    uint32_t const tsum = __reduce_add_sync(0xffffffffu, nTent);
    uint32_t const asum = __reduce_add_sync(0xffffffffu, nAcc);
    if (lane == 0) {
        tally_flush(tsum, S.stats, 1);
        tally_flush(asum, S.stats, 2);
    }
    if (tid == 0 && nAtt) atomicAdd(S.stats + (blockIdx.x % kStatSlots), nAtt);
}

// ---------------------------------------------------------------------------------- cluster-resident

// A 64-bit OR / XOR into distributed shared memory as 32-bit atomics on the two halves (the bits
// are independent, so the result is the same). Measured on B200: 64-bit bitwise atomics on
// another CTA's shared memory (through map_shared_rank, or atom.shared::cluster.*.b64) lose updates
// when several CTAs hit the same word, while 32-bit ones do not.
__device__ __forceinline__ void dsmem_or64(unsigned long long* p, unsigned long long v)
{
    unsigned int* const h = reinterpret_cast<unsigned int*>(p);
    if ((unsigned int)v) atomicOr(h, (unsigned int)v);
    if ((unsigned int)(v >> 32)) atomicOr(h + 1, (unsigned int)(v >> 32));
}
__device__ __forceinline__ void dsmem_xor64(unsigned long long* p, unsigned long long v)
{
    unsigned int* const h = reinterpret_cast<unsigned int*>(p);
    if ((unsigned int)v) atomicXor(h, (unsigned int)v);
    if ((unsigned int)(v >> 32)) atomicXor(h + 1, (unsigned int)(v >> 32));
}
__device__ __forceinline__ void dsmem_xor(unsigned int* p, unsigned int v) { atomicXor(p, v); }
__device__ __forceinline__ void dsmem_xor(unsigned long long* p, unsigned long long v) { dsmem_xor64(p, v); }

// One thread-block cluster of 2^logC CTAs (1024 threads each) owns a system whose lattice,
// temporary lattice, addresses and codes fit their shared memory together, for a whole run of
// sub-steps (layout: cluster_word_rank, cluster_slot_rank). Each CTA checks the slots it holds,
// lists its own tentative movers and performs them; lattice and temporary words and neighbours'
// codes held by another CTA are reached through distributed shared memory. Two cluster barriers
// per sub-step (after the check, after the perform) take the place of the resident kernel's CTA
// barriers; the temporary lattice has one copy per sub-step parity, each CTA clearing its words of
// the previous one while it checks. Every CTA of a cluster runs the same system and so reaches
// the same barriers. A CTA leaves only after the last barrier, when no other CTA
// accesses its shared memory any more. Grid: one cluster per system of sysList; the entries of
// sub-step t are steps[t * stride + system].
template <typename W, int K>
__global__ void __launch_bounds__(kResidentBlock, 1) k_cluster_bc(SysDev const* __restrict__ sysv,
                                                                   uint32_t const* __restrict__ sysList,
                                                                   StepEntry const* __restrict__ steps,
                                                                   uint32_t stride, uint32_t nSteps)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    uint32_t const C = cluster.num_blocks(), rank = cluster.block_rank();
    uint32_t logC = 0;
    while ((1u << logC) < C) ++logC;   // a power of two (launch_cluster_bc)
    __shared__ SysDev S;
    __shared__ uint32_t listCount[2];   // per sub-step parity
    extern __shared__ unsigned long long smem[];
    uint32_t const sysId = sysList[blockIdx.x >> logC];
    copy_desc(S, sysv + sysId);
    __syncthreads();
    uint32_t const np = S.npad, nwC = S.nwords >> logC, cap = cluster_slots_per_cta(np, logC);
    uint32_t const B = blockDim.x, tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    unsigned long long* const ptab = smem;                                   // 768 plane masks
    uint32_t* const dtab = reinterpret_cast<uint32_t*>(smem + 768);          // kDirTab words
    unsigned long long* const lat = smem + 768 + kDirTab / 2;                // nwC words
    unsigned long long* const tmp = lat + nwC;                               // 2 x nwC words
    W* const code = reinterpret_cast<W*>(tmp + 2u * nwC);                    // cap slots
    uint32_t* const pk = reinterpret_cast<uint32_t*>(code + cap);            // cap slots
    uint8_t* const mok = reinterpret_cast<uint8_t*>(pk + cap);               // 512 move-table bytes
    uint32_t* const list = reinterpret_cast<uint32_t*>(mok + 512);           // K x 1024 entries
    for (uint32_t w = tid; w < 768; w += B) ptab[w] = S.planeTab[w];
    if (tid < kDirTab) dtab[tid] = S.dirTab[tid];
    for (uint32_t w = tid; w < 512; w += B) mok[w] = S.moveOk[w];
    for (uint32_t l = tid; l < nwC; l += B) {
        lat[l] = S.lat[(l << logC) | rank];
        tmp[l] = 0ull;
        tmp[nwC + l] = 0ull;
    }
    for (uint32_t l = tid; l < cap; l += B) {
        uint32_t const g = cluster_slot_of(l, rank, logC);
        bool const in = g < np;
        code[l] = in ? *rec_code<W>(S.rec, g) : W(0);
        pk[l] = in ? *rec_pk<W>(S.rec, g) : 0u;
    }
    if (tid < 2) listCount[tid] = 0;
    cluster.sync();   // every CTA's part of the state is in place before any remote access

    auto latAt = [&](uint32_t w) { return cluster.map_shared_rank(lat + (w >> logC), w & (C - 1u)); };
    // the temporary lattice and the list count alternate with the parity of the sub-steps run, so
    // each CTA clears the previous sub-step's words while it checks: two cluster barriers per
    // sub-step (after the check, after the perform)
    auto tmpAt = [&](uint32_t par, uint32_t w) {
        return cluster.map_shared_rank(tmp + par * nwC + (w >> logC), w & (C - 1u));
    };
    auto codeAt = [&](uint32_t g) {
        return cluster.map_shared_rank(code + cluster_slot_local(g, logC), cluster_slot_rank(g, logC));
    };

    uint32_t nTent = 0, nAcc = 0;
    unsigned long long nAtt = 0;
    StepEntry next = nSteps ? steps[sysId] : StepEntry{};
    uint32_t par = 0;
    for (uint32_t t = 0; t < nSteps; ++t) {
        StepEntry const st = next;
        if (t + 1 < nSteps) next = steps[(size_t)(t + 1) * stride + sysId];   // prefetch
        if (st.color == kNoColor) continue;
        if (rank == 0) nAtt += st.cnt;
        // the previous sub-step's marks and list count: no CTA reads them after the barrier that
        // ended that sub-step, and none writes them before the barrier that ends this one
        for (uint32_t l = tid; l < nwC; l += B) tmp[(par ^ 1u) * nwC + l] = 0ull;
        if (tid == 0) listCount[par ^ 1u] = 0;
        // check: this CTA's chunks of 32 slots of the colour group (the group starts at a chunk)
        uint32_t const end = st.off + st.cnt, c0 = st.off >> 5, cEnd = (end + 31u) >> 5;
        uint32_t const cFirst = c0 + ((rank - c0) & (C - 1u));
#pragma unroll
        for (int k = 0; k < K; ++k) {
            uint32_t const c = cFirst + (warp + (uint32_t)k * 32u) * C;
            uint32_t const g = c * 32u + lane;
            bool go = false;
            uint32_t entry = 0;
            if (c < cEnd && g < end) {
                uint32_t const l = cluster_slot_local(g, logC);
                uint32_t const dir = move_dir(g - st.off, st.seed);
                uint32_t const p = pk[l];
                DirParams const D = dir_params(dtab, dir);
                if ((p & D.ma) != D.wall && bonds_ok<W, true>(code[l], dir, mok)) {
                    Plane pl;
                    front_plane<true>(pl, ptab, D, p, D.front, dir);
                    unsigned long long hit = 0ull;
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                        if (pl.m[r]) hit |= *latAt(pl.w[r]) & pl.m[r];
                    if (hit == 0ull) {
                        uint32_t const to = addr_add(p, D.ma, D.step);
                        dsmem_or64(tmpAt(par, to >> 6), 1ull << (to & 63u));
                        go = true;
                        entry = l | (dir << kSlotShift);
                    }
                }
            }
            uint32_t const bal = __ballot_sync(0xffffffffu, go);
            if (bal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&listCount[par], (uint32_t)__popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (go) list[base + __popc(bal & ((1u << lane) - 1u))] = entry;
                nTent += lane == 0 ? (uint32_t)__popc(bal) : 0u;
            }
        }
        cluster.sync();   // every CTA's marks are in place
        // perform over this CTA's list
        uint32_t const nList = listCount[par];
        for (uint32_t e = tid; e < nList; e += B) {
            uint32_t const l = list[e] & kSlotMask, dir = list[e] >> kSlotShift;
            uint32_t const g = cluster_slot_of(l, rank, logC);
            uint32_t const p = pk[l];
            uint32_t nb[CodeWord<W>::kSlots];
#pragma unroll
            for (uint32_t q = 0; q < CodeWord<W>::kSlots; ++q)
                nb[q] = q < S.maxc ? __ldg(S.nbrr + (size_t)q * np + g) : 0u;
            Plane pl;
            DirParams const D = dir_params(dtab, dir);
            front_plane<true>(pl, ptab, D, p, D.front, dir);
            unsigned long long hit = 0ull;
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (pl.m[r]) hit |= *tmpAt(par, pl.w[r]) & pl.m[r];
            if (hit != 0ull) continue;
            uint32_t const a = dir >> 1;
            int32_t const s = (dir & 1u) ? 1 : -1;
            uint32_t const p1 = addr_add(p, D.ma, D.step);
            uint32_t const w0 = p >> 6, w1 = p1 >> 6;
            if (w0 == w1) {
                dsmem_xor64(latAt(w0), (1ull << (p & 63u)) | (1ull << (p1 & 63u)));
            } else {
                dsmem_xor64(latAt(w0), 1ull << (p & 63u));
                dsmem_xor64(latAt(w1), 1ull << (p1 & 63u));
            }
            pk[l] = p1;
            image_step(S, g, a, s, p, p1, D.ma);
            W const own = code[l];
            code[l] = code_shift(own, a, -s);
            uint32_t const n = uint32_t(own >> CodeWord<W>::kCountShift) & 7u;
#pragma unroll
            for (uint32_t q = 0; q < CodeWord<W>::kSlots; ++q) {
                if (q < n) {
                    uint32_t const ent = nb[q];
                    uint32_t const cr = (0u - (uint32_t(own >> (9u * q + 3u * a)) & 7u)) & 7u;
                    uint32_t const nc = uint32_t(int32_t(cr) + s) & 7u;
                    dsmem_xor(codeAt(ent & kSlotMask), W(cr ^ nc) << (9u * (ent >> kSlotShift) + 3u * a));
                }
            }
            ++nAcc;
        }
        cluster.sync();   // every perform is done: the lattice is settled for the next check
        par ^= 1u;
    }
    // after the last cluster barrier no CTA reaches into another's shared memory
    for (uint32_t l = tid; l < nwC; l += B) S.lat[(l << logC) | rank] = lat[l];
    for (uint32_t l = tid; l < cap; l += B) {
        uint32_t const g = cluster_slot_of(l, rank, logC);
        if (g < np) {
            *rec_code<W>(S.rec, g) = code[l];
            *rec_pk<W>(S.rec, g) = pk[l];
        }
    }
    uint32_t const tsum = __reduce_add_sync(0xffffffffu, nTent);
    uint32_t const asum = __reduce_add_sync(0xffffffffu, nAcc);
    if (lane == 0) {
        tally_flush(tsum, S.stats, 1);
        tally_flush(asum, S.stats, 2);
    }
    if (tid == 0 && nAtt) atomicAdd(S.stats + (blockIdx.x % kStatSlots), nAtt);
}

// ---------------------------------------------------------------------------------- launchers

namespace {

// CTAs per SM the compiler must fit (register budget) for check / perform: shape 0 leaves the
// registers free (64 / 80), 1 asks 6 / 5 (40 / 48), 2 asks 6 / 6, 3 (the default) asks 7 / 5: the
// check at 32 registers with a 20-byte spill runs the 1024 tiles of the 256^3 melt in one wave
// (7 x 148 CTAs), 4-5 % faster than shape 1. A launch names its shape (Batch::autotune picks one);
// a negative shape means the default, which the environment variable BFM_GRID_SHAPE can change.
int default_grid_shape()
{
    static int const shape = [] {
        char const* e = std::getenv("BFM_GRID_SHAPE");
        int const v = e ? std::atoi(e) : 3;
        return (v >= 0 && v < kGridShapes) ? v : 3;
    }();
    return shape;
}

// SMs of the current device (cached per device)
int sm_count()
{
    static thread_local int count[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    int& c = count[dev & 63];
    if (!c && cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) c = 148;
    return c;
}

// the perform's warps per CTA and per tile: BFM_PERFORM_WARPS (1, 2, 4, 8) and BFM_PERFORM_GROUP
// (1, 2, 4, 8; at most the warps per CTA) override the defaults
int perform_env(char const* name, int dflt, int maxv)
{
    char const* e = std::getenv(name);
    int const v = e ? std::atoi(e) : dflt;
    return (v == 1 || v == 2 || v == 4 || v == 8) && v <= maxv ? v : dflt;
}
int perform_warps()
{
    static int const w = perform_env("BFM_PERFORM_WARPS", (int)kPerformWarpsDefault, 8);
    return w;
}
int perform_group()
{
    static int const g = std::min(perform_env("BFM_PERFORM_GROUP", (int)kPerformGroupDefault, 8), perform_warps());
    return g;
}

template <typename W, bool kMulti, int PW, int G>
void launch_perform_k(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                      StepEntry const* dSteps, PerformArgs const& pa, cudaStream_t s)
{
    uint32_t const tilesPerCta = PW / G;
    k_perform_bc<W, kMulti, PW, G><<<(nTiles + tilesPerCta - 1) / tilesPerCta, 32 * PW, 0, s>>>(
        hostDesc, dSys, dTiles, dSteps, pa.parity, pa.scope, pa.next, nTiles);
}

template <typename W, bool kMulti, int PW>
void launch_perform_g(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                      StepEntry const* dSteps, PerformArgs const& pa, cudaStream_t s)
{
    int const g = pa.group > 0 ? pa.group : perform_group();
    if (g >= 8 && PW >= 8) launch_perform_k<W, kMulti, PW, (PW >= 8 ? 8 : 1)>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s);
    else if (g >= 4 && PW >= 4) launch_perform_k<W, kMulti, PW, (PW >= 4 ? 4 : 1)>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s);
    else if (g >= 2 && PW >= 2) launch_perform_k<W, kMulti, PW, (PW >= 2 ? 2 : 1)>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s);
    else launch_perform_k<W, kMulti, PW, 1>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s);
}

template <typename W, bool kMulti, int B, int kMinCheck>
void launch_grid_bc_k(bool check, SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles,
                      uint32_t nTiles, StepEntry const* dSteps, PerformArgs const& pa, cudaStream_t s)
{
    if (check) {
        k_check_bc<W, B, kMulti, kMinCheck><<<nTiles, B, 0, s>>>(hostDesc, dSys, dTiles, dSteps, pa.snap);
        return;
    }
    switch (pa.warps > 0 ? pa.warps : perform_warps()) {
    case 1: launch_perform_g<W, kMulti, 1>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    case 2: launch_perform_g<W, kMulti, 2>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    case 8: launch_perform_g<W, kMulti, 8>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    default: launch_perform_g<W, kMulti, 4>(hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    }
}

// shape: the check's register budget in resident threads per SM, 0: the compiler's choice, 1: 1536,
// 2: 1280, 3: 1792 (the default; BFM_GRID_SHAPE overrides it); block: the check's CTA size (128, 256
// or 512 threads over the same 512-monomer tile). The perform (one warp per tile) has one form.
template <typename W, bool kMulti, int B>
void launch_grid_bc_b(bool check, SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles,
                      uint32_t nTiles, StepEntry const* dSteps, PerformArgs const& pa, int shape, cudaStream_t s)
{
    switch (shape < 0 ? default_grid_shape() : shape) {
    case 1: launch_grid_bc_k<W, kMulti, B, 1536 / B>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    case 2: launch_grid_bc_k<W, kMulti, B, 1280 / B>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    case 3: launch_grid_bc_k<W, kMulti, B, 1792 / B>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    default: launch_grid_bc_k<W, kMulti, B, 1>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, s); break;
    }
}

template <typename W, bool kMulti>
void launch_grid_bc_m(bool check, SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles,
                      uint32_t nTiles, StepEntry const* dSteps, PerformArgs const& pa, int shape, int block,
                      cudaStream_t s)
{
    if (!check) {   // the perform's form does not depend on shape or block
        launch_grid_bc_k<W, kMulti, 256, 1>(false, hostDesc, dSys, dTiles, nTiles, dSteps, pa, s);
        return;
    }
    if (block == 128) launch_grid_bc_b<W, kMulti, 128>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape, s);
    else if (block == 512) launch_grid_bc_b<W, kMulti, 512>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape, s);
    else launch_grid_bc_b<W, kMulti, 256>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape, s);
}

template <typename W>
cudaError_t launch_grid_bc(bool check, SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles,
                           uint32_t nTiles, StepEntry const* dSteps, PerformArgs const& pa, int shape, int block,
                           cudaStream_t s)
{
    if (shape >= kGridShapes || !check_block_ok(block) || !perform_shape_ok(pa.warps, pa.group))
        return cudaErrorInvalidValue;
    if (dTiles) launch_grid_bc_m<W, true>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape, block, s);
    else launch_grid_bc_m<W, false>(check, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape, block, s);
    return cudaGetLastError();
}

}  // namespace

std::vector<TileRef> perform_tile_list(std::vector<TileRef> const& tiles)
{
    // the perform takes one tile per warp, like the check's list
    std::vector<TileRef> out(tiles);
    for (auto& t : out) t.count = 1;
    return out;
}

cudaError_t launch_check_bc(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                            StepEntry const* dSteps, uint32_t codeMode, cudaStream_t s, int shape, int block,
                            unsigned long long* snap)
{
    if (nTiles == 0) return cudaSuccess;
    if (dTiles && snap) return cudaErrorInvalidValue;   // snapshots are taken for one system only
    PerformArgs none{};
    none.snap = snap;
    if (block <= 0) block = (int)kCheckBlockDefault;
    if (codeMode == kCode32)
        return launch_grid_bc<uint32_t>(true, hostDesc, dSys, dTiles, nTiles, dSteps, none, shape, block, s);
    if (codeMode == kCode64)
        return launch_grid_bc<unsigned long long>(true, hostDesc, dSys, dTiles, nTiles, dSteps, none, shape, block, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_perform_bc(SysDev const& hostDesc, SysDev const* dSys, TileRef const* dTiles, uint32_t nTiles,
                              StepEntry const* dSteps, uint32_t codeMode, cudaStream_t s, int shape,
                              PerformArgs const& pa)
{
    if (nTiles == 0) return cudaSuccess;
    if (codeMode == kCode32)
        return launch_grid_bc<uint32_t>(false, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape,
                                        (int)kCheckBlockDefault, s);
    if (codeMode == kCode64)
        return launch_grid_bc<unsigned long long>(false, hostDesc, dSys, dTiles, nTiles, dSteps, pa, shape,
                                                  (int)kCheckBlockDefault, s);
    return cudaErrorInvalidValue;
}

namespace {

// A sweep grid of at most this many CTAs runs as one cluster (a non-portable size above 8)
constexpr uint32_t kMaxSweepCluster = 16;

template <typename W, int MPT, int kMinBlocks, int B = (int)kGridBlock>
cudaError_t launch_sweep_bc_k(SysDev const& S, StepEntry const* dSteps, uint32_t nSteps, uint32_t maxGroup,
                              GridSync* gs, bool allowCluster, cudaStream_t s, uint32_t* gridOut)
{
    // co-resident CTAs per SM and SM count, once per device and instantiation; which cluster sizes
    // can run, once per device, instantiation and size
    static thread_local int occ[64] = {}, nsm[64] = {};
    static thread_local signed char clusterOk[64][kMaxSweepCluster + 1] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!occ[dev & 63]) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[dev & 63], k_sweep_bc<W, MPT, kMinBlocks, false, B>,
                                                          B, 0);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&nsm[dev & 63], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (occ[dev & 63] < 1) return cudaErrorInvalidConfiguration;
    }
    uint32_t nTiles = (maxGroup + kBcTileSpan - 1) / kBcTileSpan;
    if (nTiles == 0) nTiles = 1;
    uint32_t const grid = std::min<uint32_t>(nTiles, (uint32_t)(occ[dev & 63] * nsm[dev & 63]));
    if (gridOut) *gridOut = grid;
    void* args[] = {const_cast<SysDev*>(&S), &dSteps, &nSteps, &nTiles, &gs};
    if (allowCluster && grid <= kMaxSweepCluster) {
        // the whole grid as one cluster, its barriers in hardware, where the device can run it
        auto kernel = k_sweep_bc<W, MPT, kMinBlocks, true, B>;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = grid;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(B);
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        signed char& ok = clusterOk[dev & 63][grid];
        if (ok == 0) {
            ok = -1;
            if (grid <= 8 || cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                                 cudaSuccess) {
                int clusters = 0;
                if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) == cudaSuccess && clusters >= 1) ok = 1;
            }
            cudaGetLastError();   // a size the device refuses is not an error of this call
        }
        if (ok == 1) return cudaLaunchKernelExC(&cfg, reinterpret_cast<void const*>(kernel), args);
    }
    return cudaLaunchCooperativeKernel(reinterpret_cast<void const*>(k_sweep_bc<W, MPT, kMinBlocks, false, B>),
                                       dim3(grid), dim3(B), args, 0, s);
}

template <typename W>
cudaError_t launch_sweep_bc_w(SysDev const& S, StepEntry const* dSteps, uint32_t nSteps, uint32_t maxGroup,
                              GridSync* gs, bool allowCluster, int shape, cudaStream_t s, uint32_t* gridOut)
{
    switch (shape) {
    case 0: return launch_sweep_bc_k<W, kCheckMpt, 4>(S, dSteps, nSteps, maxGroup, gs, allowCluster, s, gridOut);
    case 1: return launch_sweep_bc_k<W, kCheckMpt, 5>(S, dSteps, nSteps, maxGroup, gs, allowCluster, s, gridOut);
    case 2: return launch_sweep_bc_k<W, kCheckMpt, 6>(S, dSteps, nSteps, maxGroup, gs, allowCluster, s, gridOut);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_sweep_bc(SysDev const& hostDesc, StepEntry const* dSteps, uint32_t nSteps, uint32_t maxGroup,
                            GridSync* gs, uint32_t codeMode, int shape, bool allowCluster, cudaStream_t s,
                            uint32_t* gridOut)
{
    if (nSteps == 0) return cudaSuccess;
    if (codeMode == kCode32)
        return launch_sweep_bc_w<uint32_t>(hostDesc, dSteps, nSteps, maxGroup, gs, allowCluster, shape, s, gridOut);
    if (codeMode == kCode64)
        return launch_sweep_bc_w<unsigned long long>(hostDesc, dSteps, nSteps, maxGroup, gs, allowCluster, shape, s,
                                                     gridOut);
    return cudaErrorInvalidValue;
}

size_t resident_bc_smem_bytes(uint32_t nwords, uint32_t npad, uint32_t maxGroup, uint32_t codeMode)
{
    size_t const w = codeMode == kCode64 ? 8 : 4;
    return 768 * 8 + kDirTab * 4 + (size_t)nwords * 3 * 8 + (size_t)npad * (w + 4) + 512 + (size_t)maxGroup * 4;
}

namespace {

template <typename W, int K>
cudaError_t launch_resident_bc_k(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, StepEntry const* dSteps,
                                 uint32_t nSys, uint32_t nSteps, size_t smem, cudaStream_t s)
{
    static thread_local size_t attrSet[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    size_t& have = attrSet[dev & 63];
    if (smem > have) {
        e = cudaFuncSetAttribute(k_resident_bc<W, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        have = smem;
    }
    k_resident_bc<W, K><<<nCta, kResidentBlock, smem, s>>>(dSys, dList, dSteps, nSys, nSteps);
    return cudaGetLastError();
}

template <typename W>
cudaError_t launch_resident_bc_w(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, uint32_t perThread,
                                 StepEntry const* dSteps, uint32_t nSys, uint32_t nSteps, size_t smem, cudaStream_t s)
{
    switch (perThread) {
    case 1: return launch_resident_bc_k<W, 1>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 2: return launch_resident_bc_k<W, 2>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 4: return launch_resident_bc_k<W, 4>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 8: return launch_resident_bc_k<W, 8>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    case 16: return launch_resident_bc_k<W, 16>(dSys, dList, nCta, dSteps, nSys, nSteps, smem, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_resident_bc(SysDev const* dSys, uint32_t const* dList, uint32_t nCta, uint32_t perThread,
                               StepEntry const* dSteps, uint32_t nSys, uint32_t nSteps, size_t smem, uint32_t codeMode,
                               cudaStream_t s)
{
    if (nCta == 0 || nSteps == 0) return cudaSuccess;
    if (smem > kResidentMaxSmem) return cudaErrorInvalidValue;
    if (codeMode == kCode32)
        return launch_resident_bc_w<uint32_t>(dSys, dList, nCta, perThread, dSteps, nSys, nSteps, smem, s);
    if (codeMode == kCode64)
        return launch_resident_bc_w<unsigned long long>(dSys, dList, nCta, perThread, dSteps, nSys, nSteps, smem, s);
    return cudaErrorInvalidValue;
}

size_t cluster_bc_smem_bytes(uint32_t nwords, uint32_t npad, uint32_t logC, uint32_t perThread, uint32_t codeMode)
{
    size_t const w = codeMode == kCode64 ? 8 : 4;
    size_t const cap = cluster_slots_per_cta(npad, logC);
    return 768 * 8 + kDirTab * 4 + (size_t)(nwords >> logC) * 3 * 8 + cap * (w + 4) + 512 +
           (size_t)perThread * kResidentBlock * 4;
}

namespace {

template <typename W, int K>
cudaError_t cluster_bc_config(uint32_t logC, size_t smem, cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr,
                              uint32_t nClusters, cudaStream_t s, bool& runnable)
{
    auto kernel = k_cluster_bc<W, K>;
    uint32_t const C = 1u << logC;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (C > 8) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg = {};
    cfg.gridDim = dim3(nClusters * C);
    cfg.blockDim = dim3(kResidentBlock);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg);
    runnable = e == cudaSuccess && clusters >= 1;
    return e;
}

template <typename W, int K>
cudaError_t launch_cluster_bc_k(SysDev const* dSys, uint32_t const* dList, uint32_t nClusters, uint32_t logC,
                                StepEntry const* dSteps, uint32_t stride, uint32_t nSteps, size_t smem,
                                cudaStream_t s)
{
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    bool runnable = false;
    cudaError_t e = cluster_bc_config<W, K>(logC, smem, cfg, attr, nClusters, s, runnable);
    if (e != cudaSuccess) return e;
    if (!runnable) return cudaErrorInvalidConfiguration;
    return cudaLaunchKernelEx(&cfg, k_cluster_bc<W, K>, dSys, dList, dSteps, stride, nSteps);
}

template <typename W>
cudaError_t launch_cluster_bc_w(SysDev const* dSys, uint32_t const* dList, uint32_t nClusters, uint32_t logC,
                                uint32_t perThread, StepEntry const* dSteps, uint32_t stride, uint32_t nSteps,
                                size_t smem, cudaStream_t s)
{
    switch (perThread) {
    case 1: return launch_cluster_bc_k<W, 1>(dSys, dList, nClusters, logC, dSteps, stride, nSteps, smem, s);
    case 2: return launch_cluster_bc_k<W, 2>(dSys, dList, nClusters, logC, dSteps, stride, nSteps, smem, s);
    case 4: return launch_cluster_bc_k<W, 4>(dSys, dList, nClusters, logC, dSteps, stride, nSteps, smem, s);
    case 8: return launch_cluster_bc_k<W, 8>(dSys, dList, nClusters, logC, dSteps, stride, nSteps, smem, s);
    default: return cudaErrorInvalidValue;
    }
}

template <typename W>
bool cluster_bc_runnable_w(uint32_t logC, uint32_t perThread, size_t smem)
{
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    bool runnable = false;
    cudaError_t e = cudaErrorInvalidValue;
    switch (perThread) {
    case 1: e = cluster_bc_config<W, 1>(logC, smem, cfg, attr, 1, nullptr, runnable); break;
    case 2: e = cluster_bc_config<W, 2>(logC, smem, cfg, attr, 1, nullptr, runnable); break;
    case 4: e = cluster_bc_config<W, 4>(logC, smem, cfg, attr, 1, nullptr, runnable); break;
    case 8: e = cluster_bc_config<W, 8>(logC, smem, cfg, attr, 1, nullptr, runnable); break;
    default: break;
    }
    if (e != cudaSuccess) cudaGetLastError();   // a configuration the device refuses is an answer, not an error
    return e == cudaSuccess && runnable;
}

}  // namespace

bool cluster_bc_runnable(uint32_t logC, uint32_t perThread, size_t smem, uint32_t codeMode)
{
    if (logC < 1 || logC > 4 || smem > kResidentMaxSmem) return false;
    if (codeMode == kCode32) return cluster_bc_runnable_w<uint32_t>(logC, perThread, smem);
    if (codeMode == kCode64) return cluster_bc_runnable_w<unsigned long long>(logC, perThread, smem);
    return false;
}

cudaError_t launch_cluster_bc(SysDev const* dSys, uint32_t const* dList, uint32_t nClusters, uint32_t logC,
                              uint32_t perThread, StepEntry const* dSteps, uint32_t stride, uint32_t nSteps,
                              size_t smem, uint32_t codeMode, cudaStream_t s)
{
    if (nClusters == 0 || nSteps == 0) return cudaSuccess;
    if (logC < 1 || logC > 4 || smem > kResidentMaxSmem) return cudaErrorInvalidValue;
    if (codeMode == kCode32)
        return launch_cluster_bc_w<uint32_t>(dSys, dList, nClusters, logC, perThread, dSteps, stride, nSteps, smem, s);
    if (codeMode == kCode64)
        return launch_cluster_bc_w<unsigned long long>(dSys, dList, nClusters, logC, perThread, dSteps, stride, nSteps,
                                                       smem, s);
    return cudaErrorInvalidValue;
}

}  // namespace bfm
