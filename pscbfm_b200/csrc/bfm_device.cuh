// Device-side types and helpers of the BFM sweep engine (sm_100a).
//
// Layout in HBM, per system (all in the colour-sorted order of the monomers):
//   x, y, z      int32 structure-of-arrays, unfolded corner positions, npad entries
//   nbr          uint32 [maxc][npad] neighbour slots (sorted ids), slot k of monomer g at k*npad+g
//   nnb          uint8  [npad] neighbour count
//   flags        uint8  [npad] tentative-move flag of the last check: dir<<2 | 1 (gather kernels)
//   tmark        uint32 [2][npad] temporary-lattice bit set by the last check of each parity
//                (word<<6 | bit, or kNoMark), used to scrub that bit one sub-step later (gather)
//   lat          uint64 occupancy words, one bit per lattice cell (the monomer's corner cell)
//   tmp          uint64 [2][nwords] ping-pong temporary lattices of tentative targets
// A 64-bit word holds one 4x4x4 brick of cells, bit (x&3) + 4 (y&3) + 16 (z&3), so the three
// cells of a front-plane row along any axis are one bit run with a fixed stride; bricks are
// numbered by the Z-curve (Morton order) of the brick coordinates, with the bits above the
// smallest axis's brick count laid out linearly (non-cubic boxes), through per-axis contribution
// tables (brickTab). The reference keeps one Z-curve index per cell (src/pscbfm/CRITICAL.cu:13-34);
// only the occupancy of each cell matters to the sweep, so the bit order inside a word is free.
// Bond-code representation (codeMode != kCodeNone) adds, per monomer, the lattice address of its
// corner (pk = brick word << 6 | bit in the brick, see lattice_address) and a word of bond-table
// indices (code), see CodeWord below, and per parity the mover lists of the grid kernels (mlist,
// mword, mcount) in place of flags and tmark.
#pragma once

#include <cstdint>

namespace bfm {

constexpr uint32_t kNoMark = 0xFFFFFFFFu;
constexpr uint32_t kNoColor = 0xFFFFFFFFu;
constexpr int kMaxConn = 16;
// Move counters: stats[c * kStatSlots + s], c = 0 attempted, 1 tentative, 2 accepted; each CTA
// adds its tally to slot blockIdx.x % kStatSlots, so no single address takes more than a few
// dozen atomics per launch. Readers sum the slots.
constexpr uint32_t kStatSlots = 64;
constexpr size_t kStatBytes = 3 * kStatSlots * sizeof(unsigned long long);

// Per-CTA tally: one shared-memory atomic per warp, one global atomic per CTA.
__device__ __forceinline__ void tally_warp(bool pred, uint32_t* ctaTally)
{
    uint32_t const b = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31u) == 0 && b) atomicAdd(ctaTally, (uint32_t)__popc(b));
}
__device__ __forceinline__ void tally_flush(uint32_t count, unsigned long long* stats, uint32_t which)
{
    if (count) atomicAdd(stats + which * kStatSlots + (blockIdx.x % kStatSlots), (unsigned long long)count);
}

// Per-slot state of the bond-code representation, one record per slot so that the check reads
// it with one load and the perform writes it with one store: the lattice address of the corner
// (pk: brick word << 6 | bit, lattice_address) and the bond-code word (CodeWord). 3 fields
// (uint32 code): {pk, code} in 8 bytes; 6 fields (uint64 code): {pk, 0, code} in 16 bytes.
template <typename W>
struct SlotRec;
template <>
struct SlotRec<uint32_t> {
    using V = uint2;
    static constexpr uint32_t kWords = 2;
};
template <>
struct SlotRec<unsigned long long> {
    using V = uint4;
    static constexpr uint32_t kWords = 4;
};
// 32-bit words per record of a code mode
__host__ __device__ __forceinline__ uint32_t rec_words(uint32_t codeMode) { return codeMode == 2u ? 4u : 2u; }

// x, y, z: the unfolded corner positions (gather representation). With bond codes they hold each
// slot's image offsets instead: the unfolded coordinate minus the coordinate inside the lattice
// (a multiple of the lattice side, zero along a walled axis), since the lattice address pk already
// holds the rest; a move changes them only when it wraps a periodic axis (slot_coord).
struct SysDev {
    int32_t* x;
    int32_t* y;
    int32_t* z;
    uint32_t const* nbr;
    uint8_t const* nnb;
    uint8_t* flags;                  // [2][npad]; the gather kernels use the first npad (unused by bond codes)
    uint32_t* tmark;                 // [2][npad] (gather kernels)
    unsigned long long* lat;
    unsigned long long* tmp;         // [2][nwords]
    uint32_t const* brickTab;        // [nb0 + nb1 + nb2]
    uint32_t const* grp;             // [2 * nColors]: offset, size
    unsigned long long* stats;       // [3][kStatSlots]: attempted, tentative, accepted (striped)
    // bond-code representation (codeMode != kCodeNone)
    uint32_t* rec;                   // [npad] records {lattice address, bond code} (SlotRec, rec_words each)
    uint32_t const* nbrr;            // [maxc][npad] neighbour slot | reverse slot << 28
    unsigned long long const* planeTab;   // [3][64][4] front-plane masks (see plane_table_fill)
    uint8_t const* moveOk;           // [512] bit d: a bond with this index stays allowed after move d
    uint32_t const* dirTab;          // [kDirTab] lattice-address parameters per direction (dir_table_fill)
    uint32_t* mlist;                 // [2][listStride] tentative movers per tile segment, per parity
    uint32_t* mword;                 // [2][listStride] each listed mover's target address (the cell it marked)
    uint32_t* mcount;                // [2][countStride] entries of each segment
    uint32_t listStride, countStride;
    uint32_t codeMode;               // kCodeNone, kCode32, kCode64
    uint32_t walls;                  // bit a: axis a is not periodic (corners stay in [0, L-2])
    uint32_t npad, nwords, maxc, nColors;
    struct StepGen* gen;             // device-side producer of the counter stream's sub-step entries
    uint32_t mask[3];                // lattice side - 1 (a power of two; the box side but along a
                                     // walled axis whose side is not one)
    uint32_t lim[3];                 // box side - 1: on a walled axis a moved corner stays below it
    uint32_t nb[3];                  // bricks per axis
    uint32_t mb, hx, hy;             // brick_index parameters
    uint32_t amask[3];               // bond codes: the lattice-address bits of each axis (axis_address_mask)
    uint32_t forbid[16];             // bit i set <=> bond index i is forbidden
};

// Grid-wide barrier of the persistent sweep kernel: a count of arrivals that only grows during a
// launch (the host zeroes it before every launch); barrier k of a launch completes when the count
// reaches k x the grid size.
struct GridSync {
    unsigned int count;   // arrivals so far in this launch
    unsigned int fault;   // set when a wait ran out; every CTA then leaves and the host reports it
    unsigned int where;   // the barrier (1, 2, ... within the launch) at which the first wait ran out
};

// Bond codes: field k (9 bits at 9k) of a monomer's code word is the bond index of
// (neighbour k - monomer), i.e. the reference's table index (CRITICAL.cu:243-261) of that bond;
// the count of fields sits above them. Valid only with symmetric neighbour lists, where the
// reverse slot of every bond exists and bonded monomers never share a colour.
constexpr uint32_t kCodeNone = 0, kCode32 = 1, kCode64 = 2;
static_assert(kCode64 == 2u, "rec_words names the 64-bit code mode by its value");
template <typename W>
struct CodeWord;
template <>
struct CodeWord<uint32_t> {
    static constexpr uint32_t kSlots = 3, kCountShift = 27;
};
template <>
struct CodeWord<unsigned long long> {
    static constexpr uint32_t kSlots = 6, kCountShift = 54;
};
constexpr uint32_t kSlotShift = 28;          // nbrr: reverse slot in the top 4 bits
constexpr uint32_t kSlotMask = (1u << kSlotShift) - 1u;

// One sub-step of one system inside a launch. color == kNoColor: the system idles.
// prevColor: colour group whose temporary-lattice marks (parity ^ 1) are scrubbed in this
// sub-step (kNoColor: nothing to scrub). off/cnt and poff/pcnt: first slot and size of the
// current and of the previous colour group (0 when absent).
struct StepEntry {
    uint32_t color;
    uint32_t seed;
    uint32_t parity;
    uint32_t prevColor;
    uint32_t off, cnt, poff, pcnt;
};

// Counter draw stream: draw k of seed s is the upper 32 bits of SplitMix64(SplitMix64(s) +
// (k + 1) * golden gamma) (Steele, Lea & Flood 2014); sub-step t consumes draws 2t (its colour,
// draw % nColors) and 2t + 1 (its seed), the reference's order (CRITICAL.cu:509-510).
__host__ __device__ __forceinline__ uint64_t sm64_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint32_t counter_draw(uint64_t seed, uint64_t k)
{
    return (uint32_t)(sm64_mix(sm64_mix(seed) + (k + 1) * 0x9E3779B97F4A7C15ull) >> 32);
}

// Device-side producer of sub-step entries for the counter stream (one per system, in its arena).
// A perform launch given a `next` slot writes the entry of sub-step `next` there (on != 0): its
// colour and seed from the counter stream of `seed`, its previous colour = the colour of sub-step
// next - 1, the one the launch performs; then it advances `next`. Consecutive launches of a
// captured graph so hand each other their entries without a host copy.
struct StepGen {
    unsigned long long seed;
    unsigned long long next;   // sub-step index of the next entry to write
    uint32_t on;               // 0: the host supplies the entries (another draw stream)
    uint32_t nColors;
    uint32_t pad[2];
};
static_assert(sizeof(StepGen) == sizeof(StepEntry), "StepGen takes one entry slot before the entries");

// Written by one thread: the entry of sub-step g->next into *out (see StepGen). s: *g as the
// caller loaded it (ahead of other work, so that its latency overlaps that work).
__device__ __forceinline__ void write_next_step(StepGen* g, StepGen const& s, uint32_t const* grp, StepEntry* out)
{
    if (!s.on) return;
    uint64_t const t = s.next;
    uint32_t const c = counter_draw(s.seed, 2 * t) % s.nColors;
    uint32_t const pc = counter_draw(s.seed, 2 * (t - 1)) % s.nColors;
    StepEntry e;
    e.color = c;
    e.seed = counter_draw(s.seed, 2 * t + 1);
    e.parity = (uint32_t)(t & 1u);
    e.prevColor = pc;
    e.off = grp[2 * c];
    e.cnt = grp[2 * c + 1];
    e.poff = grp[2 * pc];
    e.pcnt = grp[2 * pc + 1];
    *out = e;
    g->next = t + 1;
}

// Counter snapshots of graph replays: a device ring of kSnapRing slots of four words
// {attempted, tentative, accepted, sequence}; `seq` counts the snapshots taken so far.
constexpr uint32_t kSnapRing = 64;

// One warp: the sums of the three striped move counters into ring slot *seq % kSnapRing with the
// sequence number *seq + 1, then ++*seq. The caller orders every counter update before it.
__device__ __forceinline__ void snapshot_stats(unsigned long long const* stats, unsigned long long* ring,
                                               unsigned long long* seq)
{
    static_assert(kStatSlots == 64, "two slots per lane and counter");
    uint32_t const lane = threadIdx.x & 31u;
    unsigned long long const q = *seq;
    unsigned long long* const slot = ring + 4ull * (q % kSnapRing);
    unsigned long long v[3];
#pragma unroll
    for (uint32_t c = 0; c < 3; ++c)   // the six loads go out together
        v[c] = __ldcg(stats + c * kStatSlots + lane) + __ldcg(stats + c * kStatSlots + 32 + lane);
#pragma unroll
    for (uint32_t c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
        if (lane == 0) slot[c] = v[c];
    }
    if (lane == 0) {
        slot[3] = q + 1;
        *seq = q + 1;
    }
}

// Move-direction hash, src/pscbfm/CRITICAL.cu:2-11 (Jenkins' 6-shift 32-bit integer hash).
// The constants and shifts must stay as they are: they define the trajectory.
__host__ __device__ __forceinline__ uint32_t move_hash(uint32_t a)
{
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}

// Direction of the monomer with in-colour index iLocal, CRITICAL.cu:321-323.
// 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z (UpdaterGPUScBFM_AB_Type.cu:534-545).
__device__ __forceinline__ uint32_t move_dir(uint32_t iLocal, uint32_t seed)
{
    return move_hash(move_hash(iLocal) ^ seed) % 6u;
}


// Position of value v (0..3) of axis a inside a brick word: bit = x + 4 y + 16 z.
// CRITICAL.cu:334-341 (the reference's NONPERIODICITY build): along an axis with walls the moved
// corner must stay in [0, L-2]; c is the current coordinate along the move's axis (in the box on
// such an axis), and the unsigned compare against lim = L - 1 rejects both -1 and L-1.
__host__ __device__ __forceinline__ bool wall_blocks(uint32_t walls, uint32_t c, uint32_t dir, uint32_t const* lim)
{
    uint32_t const a = dir >> 1;
    uint32_t const c1 = c + ((dir & 1u) ? 1u : 0xFFFFFFFFu);
    return ((walls >> a) & 1u) && c1 >= lim[a];
}

__host__ __device__ __forceinline__ uint32_t brick_pos(uint32_t v, uint32_t a)
{
    return v << (2u * a);
}

__host__ __device__ __forceinline__ uint32_t brick_bit(uint32_t x, uint32_t y, uint32_t z)
{
    return (x & 3u) | ((y & 3u) << 2) | ((z & 3u) << 4);
}

// Mask of the cells with axis-a value in [lo, hi] (and the other two axes at 0): a run of
// hi-lo+1 ones with stride 4^a, shifted to lo.
__device__ __forceinline__ unsigned long long range_mask(uint32_t lo, uint32_t hi, uint32_t a)
{
    uint32_t const n = hi - lo;   // 0..2
    unsigned long long const rep = a == 0 ? (n == 0 ? 0x1ull : n == 1 ? 0x3ull : 0x7ull)
                                 : a == 1 ? (n == 0 ? 0x1ull : n == 1 ? 0x11ull : 0x111ull)
                                          : (n == 0 ? 0x1ull : n == 1 ? 0x10001ull : 0x100010001ull);
    return rep << (lo << (2u * a));
}

// Spreads the low 8 bits of v to every third bit (published "Part1By2" bit-interleave masks).
__host__ __device__ __forceinline__ uint32_t dilate3(uint32_t v)
{
    v &= 0xFFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Brick (word) index of brick coordinates (bx, by, bz): the low `mb` bits of the three
// coordinates interleaved as a Z-curve, the remaining high bits (non-cubic boxes) appended in
// x-fastest order; hx, hy are the high-part extents in x and y.
__host__ __device__ __forceinline__ uint32_t brick_index(uint32_t bx, uint32_t by, uint32_t bz, uint32_t mb,
                                                         uint32_t hx, uint32_t hy)
{
    uint32_t const lm = (1u << mb) - 1u;
    uint32_t const lo = dilate3(bx & lm) | (dilate3(by & lm) << 1) | (dilate3(bz & lm) << 2);
    uint32_t const hi = (bx >> mb) + hx * ((by >> mb) + hy * (bz >> mb));
    return lo | (hi << (3u * mb));
}

// Host: brick_index parameters of a box with nb[a] bricks per axis (powers of two), and the
// per-axis contributions to it (tab[0..nb0) for x, then y, then z; the index of a brick is the
// sum of its three contributions). The table-driven kernels and the arithmetic ones agree.
inline void brick_params(uint32_t const nb[3], uint32_t& mb, uint32_t& hx, uint32_t& hy)
{
    uint32_t lb[3];
    for (int a = 0; a < 3; ++a) {
        lb[a] = 0;
        while ((1u << lb[a]) < nb[a]) ++lb[a];
    }
    mb = lb[0] < lb[1] ? (lb[0] < lb[2] ? lb[0] : lb[2]) : (lb[1] < lb[2] ? lb[1] : lb[2]);
    hx = nb[0] >> mb;
    hy = nb[1] >> mb;
}

inline void brick_tables_fill(uint32_t const nb[3], uint32_t* tab)
{
    uint32_t mb, hx, hy;
    brick_params(nb, mb, hx, hy);
    for (uint32_t b = 0; b < nb[0]; ++b) tab[b] = brick_index(b, 0, 0, mb, hx, hy);
    for (uint32_t b = 0; b < nb[1]; ++b) tab[nb[0] + b] = brick_index(0, b, 0, mb, hx, hy);
    for (uint32_t b = 0; b < nb[2]; ++b) tab[nb[0] + nb[1] + b] = brick_index(0, 0, b, mb, hx, hy);
}

// Host: masks of the front plane inside the (at most 2x2) bricks it touches. Entry
// ((a*64 + lo)*4 + k) for a move along axis a, lo = the low six bits of the lattice address of the
// plane's first cell (its in-brick position: x&3 | (y&3)<<2 | (z&3)<<4): the plane lies at that
// cell's coordinate along a and spans three cells from it along the two other axes u < v;
// k = 2*i + j selects the brick (i: u-brick 0 or 1, j: v-brick 0 or 1). A run that starts at 2 or
// 3 spills into the next brick; a zero mask means that brick is not touched.
inline void plane_table_fill(unsigned long long* t)
{
    auto run = [](uint32_t ax, uint32_t lo, uint32_t hi) {
        unsigned long long m = 0;
        for (uint32_t v = lo; v <= hi; ++v) m |= 1ull << brick_pos(v, ax);
        return m;
    };
    for (uint32_t a = 0; a < 3; ++a) {
        uint32_t const u = a == 0 ? 1u : 0u, v = a == 2 ? 1u : 2u;
        for (uint32_t lo = 0; lo < 64; ++lo) {
            uint32_t const fo = (lo >> (2 * a)) & 3u, lu = (lo >> (2 * u)) & 3u, lv = (lo >> (2 * v)) & 3u;
            unsigned long long const mu0 = lu <= 1 ? run(u, lu, lu + 2) : run(u, lu, 3);
            unsigned long long const mu1 = lu <= 1 ? 0ull : run(u, 0, lu - 2);
            unsigned long long const mv0 = lv <= 1 ? run(v, lv, lv + 2) : run(v, lv, 3);
            unsigned long long const mv1 = lv <= 1 ? 0ull : run(v, 0, lv - 2);
            uint32_t const sh = brick_pos(fo, a);
            unsigned long long* e = t + (a * 64 + lo) * 4;
            e[0] = (mu0 * mv0) << sh;
            e[1] = (mu0 * mv1) << sh;
            e[2] = (mu1 * mv0) << sh;
            e[3] = (mu1 * mv1) << sh;
        }
    }
}

// Lattice address of the corner cell (x, y, z) (coordinates inside the box): its brick word << 6
// | its bit in the brick. The brick index scatters the bits of each axis's brick coordinate to
// fixed positions, so every axis owns a fixed set of address bits (axis_address_mask) and a step
// along one axis is an add confined to those bits: with M the axis's mask and D a step scattered
// into M (one cell: the lowest bit of M; minus one cell: M itself), the stepped address is
// (((p | ~M) + D) & M) | (p & ~M) — the set bits outside M carry across them, and the carry out of
// the top of M is dropped, which wraps the axis periodically.
inline uint32_t lattice_address(uint32_t x, uint32_t y, uint32_t z, uint32_t const nb[3], uint32_t const* tab)
{
    uint32_t const w = tab[x >> 2] + tab[nb[0] + (y >> 2)] + tab[nb[0] + nb[1] + (z >> 2)];
    return (w << 6) | brick_bit(x, y, z);
}

inline uint32_t axis_address_mask(uint32_t a, uint32_t const nb[3], uint32_t const* tab)
{
    uint32_t const off = a == 0 ? 0u : (a == 1 ? nb[0] : nb[0] + nb[1]);
    return (tab[off + nb[a] - 1u] << 6) | (3u << (2u * a));
}

// Per-direction parameters of the lattice-address arithmetic, kDirWords words per direction d
// (axis a = d >> 1, the two other axes u < v), stored as two arrays of 16-byte halves: words 0-3
// of direction d at 4 d, words 4-7 at kDirHalf + 4 d (kDirTab words in all). A warp's 16-byte
// loads of the six directions then fall in distinct shared-memory banks.
//   [0] Ma                     address mask of the move's axis
//   [1] step                   the move, scattered into Ma (+1 or -1 along a)
//   [2] Mu  [3] Mv             address masks of the two other axes
//   [4] front                  the front plane's offset along a, scattered into Ma (+2 or -2)
//   [5] Mu >> 6  [6] Mv >> 6   the masks of u and v in a brick index
//   [7] wall                   address bits (in Ma) of the corner that may not move along d on a
//                              walled axis (coordinate L-2 for +, 0 for -); 1 << 31 (never equal to
//                              an address's bits in Ma) when the axis is periodic
constexpr uint32_t kDirWords = 8;
constexpr uint32_t kDirHalf = 6 * 4;
constexpr uint32_t kDirTab = 6 * kDirWords;
constexpr uint32_t kNoWall = 1u << 31;

// hi[a]: the highest corner coordinate a walled axis a allows (its box side - 2); the wall word of a
// move along a walled axis is the address of the corner that may not move further that way.
inline void dir_table_fill(uint32_t const nb[3], uint32_t const* tab, uint32_t const hi[3], uint32_t walls,
                           uint32_t* out)
{
    uint32_t M[3];
    for (uint32_t a = 0; a < 3; ++a) M[a] = axis_address_mask(a, nb, tab);
    for (uint32_t d = 0; d < 6; ++d) {
        uint32_t const a = d >> 1, u = a == 0 ? 1u : 0u, v = a == 2 ? 1u : 2u;
        bool const up = (d & 1u) != 0;
        uint32_t* e = out + d * 4;
        uint32_t* f = out + kDirHalf + d * 4;
        e[0] = M[a];
        e[1] = up ? (1u << (2u * a)) : M[a];
        e[2] = M[u];
        e[3] = M[v];
        f[0] = up ? (2u << (2u * a)) : (M[a] & ~(1u << (2u * a)));   // -2: every bit of Ma but the lowest
        f[1] = M[u] >> 6;
        f[2] = M[v] >> 6;
        uint32_t c[3] = {0u, 0u, 0u};
        c[a] = up ? hi[a] : 0u;
        f[3] = ((walls >> a) & 1u) ? lattice_address(c[0], c[1], c[2], nb, tab) : kNoWall;
    }
}

struct Plane {
    uint32_t w[4];
    unsigned long long m[4];
    uint32_t touch;   // bit k set <=> brick k is touched (m[k] != 0), from the address alone
};

// Cluster-resident layout (k_cluster_bc): a system held in the shared memory of a cluster of
// 2^logC CTAs. Lattice word w (occupancy and temporary) lives in CTA w mod 2^logC at local word
// w >> logC. Slots are dealt out in chunks of 32 (a colour group starts at a multiple of 32): slot
// g lives in CTA (g / 32) mod 2^logC, at local index (g / (32 * 2^logC)) * 32 + g mod 32, so every
// colour group spreads evenly over the CTAs and a CTA checks exactly the slots it holds.
__host__ __device__ __forceinline__ uint32_t cluster_word_rank(uint32_t w, uint32_t logC)
{
    return w & ((1u << logC) - 1u);
}
__host__ __device__ __forceinline__ uint32_t cluster_word_local(uint32_t w, uint32_t logC) { return w >> logC; }
__host__ __device__ __forceinline__ uint32_t cluster_slot_rank(uint32_t g, uint32_t logC)
{
    return (g >> 5) & ((1u << logC) - 1u);
}
__host__ __device__ __forceinline__ uint32_t cluster_slot_local(uint32_t g, uint32_t logC)
{
    return ((g >> (5u + logC)) << 5) | (g & 31u);
}
// the slot held at local index l of CTA r (inverse of the two above)
__host__ __device__ __forceinline__ uint32_t cluster_slot_of(uint32_t l, uint32_t r, uint32_t logC)
{
    return ((((l >> 5) << logC) | r) << 5) | (l & 31u);
}
// local slot capacity of each CTA for npad slots (npad a multiple of 32)
__host__ __device__ __forceinline__ uint32_t cluster_slots_per_cta(uint32_t npad, uint32_t logC)
{
    uint32_t const chunks = npad >> 5;
    return ((chunks + (1u << logC) - 1u) >> logC) << 5;
}

// Per-direction parameters of the lattice-address arithmetic (dir_table_fill); the kernels read
// them from the CTA's shared copy of the table.
struct DirParams {
    uint32_t ma, step, mu, mv, front, bu, bv, wall;   // the order of dir_table_fill
};

__host__ __device__ __forceinline__ DirParams dir_params(uint32_t const* dtab, uint32_t dir)
{
    uint4 const a = *reinterpret_cast<uint4 const*>(dtab + dir * 4u);
    uint4 const b = *reinterpret_cast<uint4 const*>(dtab + kDirHalf + dir * 4u);
    return {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

// The lattice address p stepped by d, scattered into the axis mask m (see lattice_address).
__host__ __device__ __forceinline__ uint32_t addr_add(uint32_t p, uint32_t m, uint32_t d)
{
    return (((p | ~m) + d) & m) | (p & ~m);
}

// The scattered step opposite to step along the axis with mask ma: -1 (ma) for a positive move,
// +1 (the lowest bit of ma) for a negative one.
__host__ __device__ __forceinline__ uint32_t addr_back(uint32_t ma, uint32_t step)
{
    return step ^ ma ^ (ma & (0u - ma));
}

// Coordinate along an axis of the lattice address p: the address bits under the axis's mask m,
// packed in order (an axis's bits keep their significance in the address). A bit-by-bit extract,
// for read-back and set-up, not for the sweep.
__host__ __device__ __forceinline__ uint32_t axis_coord(uint32_t p, uint32_t m)
{
    uint32_t r = 0u, bit = 1u;
    while (m) {
        uint32_t const low = m & (0u - m);
        if (p & low) r |= bit;
        bit <<= 1;
        m ^= low;
    }
    return r;
}

// Image offset of an unfolded coordinate c on an axis of lattice side P (a power of two): c minus
// its coordinate inside the lattice, i.e. c with its low log2(P) bits cleared.
__host__ __device__ __forceinline__ int32_t image_offset(int32_t c, uint32_t P)
{
    return int32_t(uint32_t(c) & ~(P - 1u));
}

// Unfolded coordinate along axis a of slot g (padding slots keep kPadCoord in x): with bond codes
// the image offset in x/y/z plus the coordinate read from the lattice address.
__device__ __forceinline__ int32_t slot_coord(SysDev const& S, uint32_t g, uint32_t a)
{
    int32_t const* const X = a == 0 ? S.x : (a == 1 ? S.y : S.z);
    int32_t const off = X[g];
    if (S.codeMode == kCodeNone) return off;
    return off + int32_t(axis_coord(S.rec[(size_t)g * rec_words(S.codeMode)], S.amask[a]));
}

// The lattice address and the bond-code word of slot g inside its record.
template <typename W>
__host__ __device__ __forceinline__ uint32_t* rec_pk(uint32_t* r, uint32_t g)
{
    return r + (size_t)g * SlotRec<W>::kWords;
}
template <typename W>
__host__ __device__ __forceinline__ W* rec_code(uint32_t* r, uint32_t g)
{
    return reinterpret_cast<W*>(r + (size_t)g * SlotRec<W>::kWords + SlotRec<W>::kWords / 2);
}
// The code word of a record as loaded (V: uint2 or uint4).
__host__ __device__ __forceinline__ uint32_t rec_code_of(uint2 v) { return v.y; }
__host__ __device__ __forceinline__ unsigned long long rec_code_of(uint4 v)
{
    return v.z | ((unsigned long long)v.w << 32);
}
// A record with address p and code word c.
__host__ __device__ __forceinline__ uint2 make_rec(uint32_t p, uint32_t c) { return make_uint2(p, c); }
__host__ __device__ __forceinline__ uint4 make_rec(uint32_t p, unsigned long long c)
{
    return make_uint4(p, 0u, uint32_t(c), uint32_t(c >> 32));
}

// The <= 2x2 brick words of the front plane of a move along dir and their masks. The plane's
// first cell is base + da along the move's axis (da scattered into Ma) and -1 along the two other
// axes: da = D.front (+2 d) from the monomer's address, D.step (+d) from its target's; the low
// six bits of its address select the masks (ptab: global memory through L1, or shared memory)
// and the neighbouring bricks along u and v are one step of the brick index along those axes.
template <bool kSharedTables>
__host__ __device__ __forceinline__ void front_plane(Plane& pl, unsigned long long const* ptab, DirParams const& D,
                                                     uint32_t base, uint32_t da, uint32_t dir)
{
    uint32_t const f = ((((base | ~D.ma) + da) & D.ma) | (((base | ~D.mu) + D.mu) & D.mu)) |
                       (((base | ~D.mv) + D.mv) & D.mv);
    uint32_t const ti = ((dir >> 1) * 64u + (f & 63u)) * 4u;
    ulonglong2 m01, m23;
#ifdef __CUDA_ARCH__
    if (!kSharedTables) {
        m01 = __ldg(reinterpret_cast<ulonglong2 const*>(ptab + ti));
        m23 = __ldg(reinterpret_cast<ulonglong2 const*>(ptab + ti + 2));
    } else
#endif
    {
        m01 = *reinterpret_cast<ulonglong2 const*>(ptab + ti);
        m23 = *reinterpret_cast<ulonglong2 const*>(ptab + ti + 2);
    }
    uint32_t const w00 = f >> 6;
    uint32_t const w10 = addr_add(w00, D.bu, 1u);
    pl.w[0] = w00;
    pl.m[0] = m01.x;
    pl.w[1] = addr_add(w00, D.bv, 1u);
    pl.m[1] = m01.y;
    pl.w[2] = w10;
    pl.m[2] = m23.x;
    pl.w[3] = addr_add(w10, D.bv, 1u);
    pl.m[3] = m23.y;
    // the run of three cells along u (v) spills into the next brick when it starts at in-brick
    // coordinate 2 or 3, i.e. when the high in-brick bit of that axis (one of bits 1, 3, 5) is set;
    // loads predicated on this need not wait for the masks
    uint32_t const tu = (f & D.mu & 0x2Au) != 0u, tv = (f & D.mv & 0x2Au) != 0u;
    pl.touch = 1u | (tv << 1) | (tu << 2) | ((tu & tv) << 3);
}

// Host: bit d of ok[idx] is set when the bond with table index idx (neighbour - monomer, every
// component mod 8) is still allowed after the monomer moves along direction d.
inline void move_ok_fill(bool const* forbidden512, uint8_t* ok)
{
    for (uint32_t idx = 0; idx < 512; ++idx) {
        uint8_t m = 0;
        for (uint32_t d = 0; d < 6; ++d) {
            uint32_t const a = d >> 1;
            uint32_t const c = (idx >> (3 * a)) & 7u;
            uint32_t const nc = (c + ((d & 1u) ? 7u : 1u)) & 7u;   // neighbour - (monomer + d)
            uint32_t const j = (idx & ~(7u << (3 * a))) | (nc << (3 * a));
            if (!forbidden512[j]) m |= (uint8_t)(1u << d);
        }
        ok[idx] = m;
    }
}

// Bond-set lookup, CRITICAL.cu:243-261 + :350: index of (dx,dy,dz) with every component masked
// to 3 bits; the difference is taken in 32-bit arithmetic, which keeps the low 3 bits exact.
__device__ __forceinline__ uint32_t bond_index(int32_t dx, int32_t dy, int32_t dz)
{
    return (uint32_t(dx) & 7u) | ((uint32_t(dy) & 7u) << 3) | ((uint32_t(dz) & 7u) << 6);
}

__device__ __forceinline__ bool forbidden(uint32_t const* tbl, uint32_t idx)
{
    return (tbl[idx >> 5] >> (idx & 31u)) & 1u;
}

// Shifts component `axis` of every bond field of a code word by `delta` (mod 8). The monomer's
// own bonds change by -d when it moves by d, the reverse bond of a neighbour by +d.
template <typename W>
__device__ __forceinline__ W code_shift(W code, uint32_t axis, int32_t delta)
{
    uint32_t const n = uint32_t(code >> CodeWord<W>::kCountShift) & 7u;
    W out = code;
#pragma unroll
    for (uint32_t k = 0; k < CodeWord<W>::kSlots; ++k) {
        if (k < n) {
            uint32_t const sh = 9u * k + 3u * axis;
            uint32_t const c = uint32_t(code >> sh) & 7u;
            uint32_t const nc = uint32_t(int32_t(c) + delta) & 7u;
            out ^= W(c ^ nc) << sh;
        }
    }
    return out;
}

// True if every bond of the code word stays in the allowed set after a move along dir.
template <typename W>
__device__ __forceinline__ bool code_bonds_ok(W code, uint32_t dir, uint32_t const* tbl)
{
    uint32_t const n = uint32_t(code >> CodeWord<W>::kCountShift) & 7u;
    uint32_t const axis = dir >> 1;
    int32_t const delta = (dir & 1u) ? -1 : 1;   // neighbour - (self + d)
    bool ok = true;
#pragma unroll
    for (uint32_t k = 0; k < CodeWord<W>::kSlots; ++k) {
        if (k < n) {
            uint32_t f = uint32_t(code >> (9u * k)) & 511u;
            uint32_t const c = (f >> (3u * axis)) & 7u;
            f ^= ((c ^ (uint32_t(int32_t(c) + delta) & 7u)) << (3u * axis));
            ok = ok && !forbidden(tbl, f);
        }
    }
    return ok;
}

__device__ __forceinline__ uint32_t pack_coord(uint32_t x, uint32_t y, uint32_t z)
{
    return x | (y << 10) | (z << 20);
}

// Word index of the brick containing cell (x,y,z) (coordinates already masked into the box).
__device__ __forceinline__ uint32_t brick_word(uint32_t const* tab, uint32_t const* nb, uint32_t x, uint32_t y,
                                               uint32_t z)
{
    return tab[x >> 2] + tab[nb[0] + (y >> 2)] + tab[nb[0] + nb[1] + (z >> 2)];
}

// The 3x3 "front plane" test of CRITICAL.cu:62-176 (byte lattice) / :179-240 (bit lattice):
// true if any cell of the plane at r0 + 2*d, +-1 in the two perpendicular axes, is set.
// The 9 cells span at most 2x2 bricks; each brick is read once with a mask.
template <typename LoadWord>
__device__ __forceinline__ bool front_occupied(LoadWord load, uint32_t const* tab, uint32_t const* nb,
                                               uint32_t const* mask, int32_t x0, int32_t y0, int32_t z0,
                                               uint32_t dir)
{
    uint32_t const a = dir >> 1;
    uint32_t const u = a == 0 ? 1u : 0u;
    uint32_t const v = a == 2 ? 1u : 2u;
    auto coord = [x0, y0, z0](uint32_t ax) { return ax == 0 ? x0 : (ax == 1 ? y0 : z0); };
    int32_t const step = (dir & 1u) ? 2 : -2;
    uint32_t const f = uint32_t(coord(a) + step) & mask[a];
    uint32_t const fpos = brick_pos(f & 3u, a);
    uint32_t const fb = f >> 2;

    uint32_t const pu = uint32_t(coord(u) - 1) & mask[u];
    uint32_t const pv = uint32_t(coord(v) - 1) & mask[v];
    uint32_t const lu = pu & 3u, lv = pv & 3u;
    uint32_t const bu0 = pu >> 2, bv0 = pv >> 2;
    uint32_t const bu1 = (bu0 + 1u) & (nb[u] - 1u);
    uint32_t const bv1 = (bv0 + 1u) & (nb[v] - 1u);
    unsigned long long const mu0 = lu <= 1u ? range_mask(lu, lu + 2u, u) : range_mask(lu, 3u, u);
    unsigned long long const mu1 = lu <= 1u ? 0ull : range_mask(0u, lu - 2u, u);
    unsigned long long const mv0 = lv <= 1u ? range_mask(lv, lv + 2u, v) : range_mask(lv, 3u, v);
    unsigned long long const mv1 = lv <= 1u ? 0ull : range_mask(0u, lv - 2u, v);

    uint32_t const offA = a == 0 ? 0u : (a == 1 ? nb[0] : nb[0] + nb[1]);
    uint32_t const offU = u == 0 ? 0u : nb[0];
    uint32_t const offV = v == 1 ? nb[0] : nb[0] + nb[1];
    uint32_t const wa = tab[offA + fb];
    uint32_t const wu0 = tab[offU + bu0], wu1 = tab[offU + bu1];
    uint32_t const wv0 = tab[offV + bv0], wv1 = tab[offV + bv1];

    // Distinct axes use disjoint binary digits of the in-brick bit position, so the product of
    // two one-axis masks is the 2-D mask without carries.
    unsigned long long hit = load(wa + wu0 + wv0) & ((mu0 * mv0) << fpos);
    if (mv1) hit |= load(wa + wu0 + wv1) & ((mu0 * mv1) << fpos);
    if (mu1) {
        hit |= load(wa + wu1 + wv0) & ((mu1 * mv0) << fpos);
        if (mv1) hit |= load(wa + wu1 + wv1) & ((mu1 * mv1) << fpos);
    }
    return hit != 0ull;
}

}  // namespace bfm
