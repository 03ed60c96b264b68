// Host check (no GPU) of the lattice-address arithmetic the bond-code kernels use
// (pscbfm_b200/csrc/bfm_device.cuh). For several box shapes, every corner position and every
// direction d (axis a, sign s):
//   1. the step lands on the address of the cell one move away (periodic wrap included);
//   2. the front plane's words and masks name exactly the nine cells p + 2 s e_a + i e_u + j e_v,
//      i, j in {-1, 0, 1}: the cells whose corners the moved cube would newly overlap;
//   3. on a walled axis the wall entry blocks exactly the moves that leave [0, L-2], and on a
//      periodic axis it blocks none;
//   4. read-back: the coordinate extracted from the address (axis_coord under the axis's address
//      mask) is the coordinate, the image offset of an unfolded coordinate plus it gives the
//      unfolded coordinate back, and a move wraps the periodic axis (the image-offset update)
//      exactly when the address bits of the axis are zero after a + move or before a - move.
// Prints "ok" and exits 0, or prints the first disagreement and exits 1.
#include <cstdio>
#include <set>
#include <utility>
#include <vector>

#include "bfm_device.cuh"

using namespace bfm;

namespace {

uint32_t address(uint32_t const c[3], uint32_t const nb[3], std::vector<uint32_t> const& tab)
{
    return lattice_address(c[0], c[1], c[2], nb, tab.data());
}

int check_box(uint32_t const box[3])
{
    uint32_t const nb[3] = {box[0] / 4, box[1] / 4, box[2] / 4};
    uint32_t const mask[3] = {box[0] - 1, box[1] - 1, box[2] - 1};
    uint32_t const hi[3] = {box[0] - 2, box[1] - 2, box[2] - 2};
    std::vector<uint32_t> tab(nb[0] + nb[1] + nb[2]);
    brick_tables_fill(nb, tab.data());
    std::vector<unsigned long long> ptab(768);
    plane_table_fill(ptab.data());
    alignas(16) uint32_t dirP[kDirTab], dirW[kDirTab];
    dir_table_fill(nb, tab.data(), hi, 0u, dirP);
    dir_table_fill(nb, tab.data(), hi, 7u, dirW);
    uint32_t amask[3];
    for (uint32_t a = 0; a < 3; ++a) amask[a] = axis_address_mask(a, nb, tab.data());
    for (uint32_t z = 0; z < box[2]; ++z)
        for (uint32_t y = 0; y < box[1]; ++y)
            for (uint32_t x = 0; x < box[0]; ++x) {
                uint32_t const c0[3] = {x, y, z};
                uint32_t const p = address(c0, nb, tab);
                for (uint32_t a = 0; a < 3; ++a) {
                    if (axis_coord(p, amask[a]) != c0[a]) {
                        std::printf("axis_coord: box %u %u %u at %u %u %u axis %u\n", box[0], box[1], box[2], x, y, z, a);
                        return 1;
                    }
                    for (int32_t k = -3; k <= 3; ++k) {
                        int32_t const unfolded = int32_t(c0[a]) + k * int32_t(box[a]);
                        if (image_offset(unfolded, box[a]) + int32_t(axis_coord(p, amask[a])) != unfolded) {
                            std::printf("image offset: box %u %u %u coordinate %d axis %u\n", box[0], box[1], box[2],
                                        unfolded, a);
                            return 1;
                        }
                    }
                    DirParams const U = dir_params(dirP, 2 * a + 1);
                    bool const upWraps = (addr_add(p, U.ma, U.step) & U.ma) == 0u, downWraps = (p & U.ma) == 0u;
                    if (upWraps != (c0[a] == box[a] - 1) || downWraps != (c0[a] == 0)) {
                        std::printf("wrap test: box %u %u %u at %u %u %u axis %u\n", box[0], box[1], box[2], x, y, z, a);
                        return 1;
                    }
                }
                for (uint32_t d = 0; d < 6; ++d) {
                    uint32_t const a = d >> 1, u = a == 0 ? 1u : 0u, v = a == 2 ? 1u : 2u;
                    int32_t const s = (d & 1u) ? 1 : -1;
                    DirParams const D = dir_params(dirP, d);
                    // the perform kernel loads words 0 and 1 of an entry as (Ma, step)
                    if (dirP[d * 4] != D.ma || dirP[d * 4 + 1] != D.step) {
                        std::printf("direction table order\n");
                        return 1;
                    }
                    // 1. the step
                    uint32_t c1[3] = {x, y, z};
                    c1[a] = uint32_t(int32_t(c1[a]) + s) & mask[a];
                    if (addr_add(p, D.ma, D.step) != address(c1, nb, tab)) {
                        std::printf("step: box %u %u %u at %u %u %u dir %u\n", box[0], box[1], box[2], x, y, z, d);
                        return 1;
                    }
                    // 2. the front plane
                    Plane pl;
                    front_plane<true>(pl, ptab.data(), D, p, D.front, d);
                    // the same plane from the target's address (the grid perform's form), and the
                    // step back from the target
                    uint32_t const to = addr_add(p, D.ma, D.step);
                    Plane pt;
                    front_plane<true>(pt, ptab.data(), D, to, D.step, d);
                    for (int r = 0; r < 4; ++r)
                        if (pt.m[r] != pl.m[r] || (pl.m[r] && pt.w[r] != pl.w[r])) {
                            std::printf("plane from the target: box %u %u %u at %u %u %u dir %u\n", box[0], box[1],
                                        box[2], x, y, z, d);
                            return 1;
                        }
                    if (addr_add(to, D.ma, addr_back(D.ma, D.step)) != p) {
                        std::printf("step back: box %u %u %u at %u %u %u dir %u\n", box[0], box[1], box[2], x, y, z, d);
                        return 1;
                    }
                    for (int r = 0; r < 4; ++r)
                        if (((pl.touch >> r) & 1u) != (pl.m[r] != 0ull ? 1u : 0u) ||
                            ((pt.touch >> r) & 1u) != (pt.m[r] != 0ull ? 1u : 0u)) {
                            std::printf("touched bricks: box %u %u %u at %u %u %u dir %u\n", box[0], box[1], box[2], x,
                                        y, z, d);
                            return 1;
                        }
                    std::set<std::pair<uint32_t, uint32_t>> got, want;
                    for (int r = 0; r < 4; ++r)
                        for (uint32_t b = 0; b < 64; ++b)
                            if ((pl.m[r] >> b) & 1ull) got.insert({pl.w[r], b});
                    for (int i = -1; i <= 1; ++i)
                        for (int j = -1; j <= 1; ++j) {
                            uint32_t c[3] = {x, y, z};
                            c[a] = uint32_t(int32_t(c[a]) + 2 * s) & mask[a];
                            c[u] = uint32_t(int32_t(c[u]) + i) & mask[u];
                            c[v] = uint32_t(int32_t(c[v]) + j) & mask[v];
                            uint32_t const q = address(c, nb, tab);
                            want.insert({q >> 6, q & 63u});
                        }
                    if (got != want) {
                        std::printf("plane: box %u %u %u at %u %u %u dir %u (%zu cells, want %zu)\n", box[0], box[1],
                                    box[2], x, y, z, d, got.size(), want.size());
                        return 1;
                    }
                    // 3. walls: corners of a walled axis lie in [0, L-2]
                    if ((p & D.ma) == D.wall) {
                        std::printf("periodic axis blocked: box %u %u %u dir %u\n", box[0], box[1], box[2], d);
                        return 1;
                    }
                    if (c0[a] <= mask[a] - 1u) {
                        DirParams const W = dir_params(dirW, d);
                        int32_t const t = int32_t(c0[a]) + s;
                        bool const leaves = t < 0 || t > int32_t(mask[a]) - 1;
                        if (((p & W.ma) == W.wall) != leaves) {
                            std::printf("wall: box %u %u %u at %u %u %u dir %u\n", box[0], box[1], box[2], x, y, z, d);
                            return 1;
                        }
                    }
                }
            }
    return 0;
}

}  // namespace

int main()
{
    uint32_t const boxes[][3] = {{4, 4, 4},    {8, 8, 8},    {32, 32, 32}, {16, 32, 64},
                                 {64, 8, 4},   {128, 16, 32}, {4, 64, 8},  {8, 4, 256}};
    for (auto const& b : boxes)
        if (check_box(b)) return 1;
    // the largest box: the address uses 30 bits, and the top corner steps and wraps correctly
    uint32_t const nb[3] = {256, 256, 256};
    std::vector<uint32_t> tab(768);
    brick_tables_fill(nb, tab.data());
    uint32_t const hi[3] = {1022, 1022, 1022};
    alignas(16) uint32_t dir[kDirTab];
    dir_table_fill(nb, tab.data(), hi, 0u, dir);
    uint32_t const top[3] = {1023, 1023, 1023}, zero[3] = {0, 0, 0};
    uint32_t const pt = address(top, nb, tab);
    if (pt >= (1u << 30)) return std::printf("address of the top corner exceeds 30 bits\n"), 1;
    for (uint32_t a = 0; a < 3; ++a)
        if (axis_coord(pt, axis_address_mask(a, nb, tab.data())) != 1023u) return std::printf("axis_coord at 1023\n"), 1;
    for (uint32_t d = 1; d < 6; d += 2) {
        DirParams const D = dir_params(dir, d);
        uint32_t c[3] = {1023, 1023, 1023};
        c[d >> 1] = 0;
        if (addr_add(pt, D.ma, D.step) != address(c, nb, tab)) return std::printf("wrap at 1024\n"), 1;
        DirParams const M = dir_params(dir, d - 1);
        uint32_t e[3] = {0, 0, 0};
        e[d >> 1] = 1023;
        if (addr_add(address(zero, nb, tab), M.ma, M.step) != address(e, nb, tab)) return std::printf("wrap at 0\n"), 1;
    }
    // the cluster-resident layout: every slot and every lattice word has one owner and one local
    // index inside that owner's capacity, and the inverse maps back
    for (uint32_t logC = 1; logC <= 4; ++logC) {
        uint32_t const C = 1u << logC;
        for (uint32_t npad : {32u, 64u, 96u, 480u, 4096u, 11264u + 32u, 131072u}) {
            uint32_t const cap = cluster_slots_per_cta(npad, logC);
            std::vector<char> seen((size_t)C * cap, 0);
            for (uint32_t g = 0; g < npad; ++g) {
                uint32_t const r = cluster_slot_rank(g, logC), l = cluster_slot_local(g, logC);
                if (r >= C || l >= cap || seen[(size_t)r * cap + l] || cluster_slot_of(l, r, logC) != g)
                    return std::printf("cluster slot layout: C %u npad %u slot %u\n", C, npad, g), 1;
                seen[(size_t)r * cap + l] = 1;
            }
        }
        for (uint32_t nw : {2u, 16u, 64u, 512u, 4096u, 32768u}) {
            if (nw < C) continue;
            std::vector<char> seen(nw, 0);
            for (uint32_t w = 0; w < nw; ++w) {
                uint32_t const r = cluster_word_rank(w, logC), l = cluster_word_local(w, logC);
                if (r >= C || l >= nw / C || seen[(size_t)r * (nw / C) + l])
                    return std::printf("cluster word layout: C %u nw %u word %u\n", C, nw, w), 1;
                seen[(size_t)r * (nw / C) + l] = 1;
            }
        }
    }
    std::printf("ok\n");
    return 0;
}
