// Device-side types and helpers of the BFM sweep engine (sm_100a).
//
// Layout in HBM, per system (all in the colour-sorted order of the monomers):
//   x, y, z      int32 structure-of-arrays, unfolded corner positions, npad entries
//   nbr          uint32 [maxc][npad] neighbour slots (sorted ids), slot k of monomer g at k*npad+g
//   nnb          uint8  [npad] neighbour count
//   flags        uint8  [npad] tentative-move flag of the last check: dir<<2 | 1
//   tmark        uint32 [2][npad] temporary-lattice bit set by the last check of each parity
//                (word<<6 | bit, or kNoMark), used to scrub that bit one sub-step later
//   lat          uint64 occupancy words, one bit per lattice cell (the monomer's corner cell)
//   tmp          uint64 [2][nwords] ping-pong temporary lattices of tentative targets
// A 64-bit word holds one 4x4x4 brick of cells in Z-curve order (bit = x0 y0 z0 x1 y1 z1);
// bricks are numbered by per-axis contribution tables (brickTab), which the host fills with the
// Z-curve of the brick coordinates. For a cubic box the bit of cell (x,y,z) is then exactly the
// reference's Z-curve index (src/pscbfm/CRITICAL.cu:13-34 with USE_ZCURVE_FOR_LATTICE).
#pragma once

#include <cstdint>

namespace bfm {

constexpr uint32_t kNoMark = 0xFFFFFFFFu;
constexpr uint32_t kNoColor = 0xFFFFFFFFu;
constexpr int kMaxConn = 16;

struct SysDev {
    int32_t* x;
    int32_t* y;
    int32_t* z;
    uint32_t const* nbr;
    uint8_t const* nnb;
    uint8_t* flags;
    uint32_t* tmark;                 // [2][npad]
    unsigned long long* lat;
    unsigned long long* tmp;         // [2][nwords]
    uint32_t const* brickTab;        // [nb0 + nb1 + nb2]
    uint32_t const* grp;             // [2 * nColors]: offset, size
    unsigned long long* stats;       // [4]: attempted, tentative, accepted, spare
    uint32_t npad, nwords, maxc, nColors;
    uint32_t mask[3];                // box side - 1 (power-of-two box)
    uint32_t nb[3];                  // bricks per axis
    uint32_t forbid[16];             // bit i set <=> bond index i is forbidden
};

// One sub-step of one system inside a launch. color == kNoColor: the system idles.
// prevColor: colour group whose temporary-lattice marks (parity ^ 1) are scrubbed in this
// sub-step's perform phase (kNoColor: nothing to scrub).
struct StepEntry {
    uint32_t color;
    uint32_t seed;
    uint32_t parity;
    uint32_t prevColor;
};

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

// Position of value v (0..3) of axis a inside a brick word.
__device__ __forceinline__ uint32_t brick_pos(uint32_t v, uint32_t a)
{
    return ((v & 1u) | ((v & 2u) << 2)) << a;
}

__device__ __forceinline__ uint32_t brick_bit(uint32_t x, uint32_t y, uint32_t z)
{
    return brick_pos(x & 3u, 0) | brick_pos(y & 3u, 1) | brick_pos(z & 3u, 2);
}

// Mask of the cells with axis-a value in [lo, hi] (and the other two axes at 0).
__device__ __forceinline__ unsigned long long range_mask(uint32_t lo, uint32_t hi, uint32_t a)
{
    unsigned long long m = 0;
#pragma unroll
    for (uint32_t v = 0; v < 4; ++v)
        if (v >= lo && v <= hi) m |= 1ull << brick_pos(v, a);
    return m;
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
