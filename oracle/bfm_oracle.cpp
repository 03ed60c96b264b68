// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A single-threaded CPU restatement of the parallel sweep of pscbfm's GPU updater
// (src/pscbfm/UpdaterGPUScBFM_AB_Type.cu + src/pscbfm/CRITICAL.cu + src/pscbfm/graphColoring.tpp).
// It is the checker for the CUDA engine in pscbfm_b200/: only the tests, the smoke entry and
// the CPU-baseline leg of the benchmark load it. Nothing in the product links or calls it.
//
// Parity pin: the same functions are run against the reference updater itself, compiled for
// sm_100a from its own sources (oracle/Makefile, target `ref`) and fed the same host draw stream;
// the results are committed as golden fixtures under tests/golden/.
//
// Every function cites the reference file:line it restates.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

// ---------------------------------------------------------------- RNG pieces

// Per-move direction hash, CRITICAL.cu:2-11 (Jenkins' 6-shift 32-bit integer hash).
inline uint32_t move_hash(uint32_t a)
{
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}

// Host draw stream of the engine (counter-based, keyed by (seed, draw index)).
// SplitMix64 finaliser (Steele, Lea & Flood 2014). Sub-step t consumes draws 2t (colour) and
// 2t+1 (sub-step seed), the order of CRITICAL.cu:509-510.
inline uint64_t sm64_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint32_t counter_draw(uint64_t seed, uint64_t k)
{
    return (uint32_t)(sm64_mix(sm64_mix(seed) + (k + 1) * 0x9E3779B97F4A7C15ull) >> 32);
}

// ---------------------------------------------------------------- system

struct System {
    uint32_t n = 0;
    uint32_t box[3] = {0, 0, 0};
    std::vector<int32_t> x, y, z;                 // original monomer order
    std::vector<std::vector<uint32_t>> nbr;       // directed lists, in setConnectivity order
    bool forbidden[512];
    uint32_t walls = 0;                           // bit a: axis a is not periodic
    uint32_t lattice[3] = {0, 0, 0};              // cells per axis (see make_system)
};

// CRITICAL.cu:334-341 (build with NONPERIODICITY): along an axis with walls the moved corner must
// stay in [0, L-2] (the unsigned compare r1 < L-1 also rejects -1), so the whole cube stays inside.
inline bool outside_walls(System const& s, int32_t x1, int32_t y1, int32_t z1)
{
    int32_t const c[3] = {x1, y1, z1};
    for (int a = 0; a < 3; ++a)
        if (((s.walls >> a) & 1u) && uint32_t(c[a]) >= s.box[a] - 1u) return true;
    return false;
}

// CRITICAL.cu:243-261: bond vector -> 9-bit table index, each component masked to 3 bits.
inline uint32_t bond_index(int32_t dx, int32_t dy, int32_t dz)
{
    return (uint32_t(dx) & 7u) | ((uint32_t(dy) & 7u) << 3) | ((uint32_t(dz) & 7u) << 6);
}

// ---------------------------------------------------------------- colouring
//
// graphColoring.tpp:77-293 with bUniformColors = true (UpdaterGPUScBFM_AB_Type.cu:550).
// The std::map "first unused colour" probe at :142-148 keeps its keys contiguous from 0, so it
// returns the smallest colour not used by an already-coloured listed neighbour; colour 255 is
// reserved for "uncoloured" and reaching it throws (:88-90, :147-148).
std::vector<uint8_t> colour_graph(System const& s)
{
    const uint8_t kNone = 255;
    const int kMaxColors = 255;
    uint32_t const n = s.n;
    std::vector<uint8_t> col(n, kNone);
    std::vector<size_t> count;                     // nColorsUsed
    bool used[256];

    auto first_free = [&](uint32_t node) {
        std::fill(used, used + 256, false);
        for (uint32_t nb : s.nbr[node])
            if (col.at(nb) != kNone) used[col[nb]] = true;
        int c = 0;
        while (c < kMaxColors && used[c]) ++c;
        if (c == kMaxColors)
            throw std::runtime_error("Already used up the maximum amount of colors. Can't color the given polymer system automatically!");
        return c;
    };

    // depth-first walk of each connected molecule, graphColoring.tpp:97-212
    for (uint32_t start = 0; start < n; ++start) {
        if (col[start] != kNone) continue;
        std::vector<uint32_t> todo;                // std::stack
        long long cur = start;
        for (;;) {
            size_t nUncol = 0;
            long long firstUncol = -1;
            for (uint32_t nb : s.nbr[(size_t)cur]) {
                if (col.at(nb) == kNone) {
                    ++nUncol;
                    if (firstUncol < 0) firstUncol = nb;
                }
            }
            int const c = first_free((uint32_t)cur);
            col[(size_t)cur] = (uint8_t)c;
            if ((size_t)c >= count.size()) count.resize(c + 1, 0);
            ++count[c];

            if (nUncol == 0 && todo.empty()) break;
            if (nUncol > 1) todo.push_back((uint32_t)cur);
            cur = firstUncol;
            if (nUncol == 0) {
                // backtrack, graphColoring.tpp:170-208
                while (!todo.empty()) {
                    cur = todo.back();
                    size_t n2 = 0;
                    long long f2 = -1;
                    for (uint32_t nb : s.nbr[(size_t)cur]) {
                        if (col.at(nb) == kNone) {
                            ++n2;
                            if (f2 < 0) f2 = nb;
                        }
                    }
                    if (n2 < 2) todo.pop_back();
                    if (f2 >= 0) { cur = f2; break; }
                    cur = -1;
                }
                if (todo.empty() && cur < 0) break;
            }
        }
    }

    // uniform rebalancing, graphColoring.tpp:216-290
    std::vector<std::pair<uint8_t, size_t>> rarest(count.size());
    for (size_t i = 0; i < count.size(); ++i) rarest[i] = {(uint8_t)i, count[i]};
    // unstable sort at :224-227 (libstdc++ std::sort with the same comparator)
    std::sort(rarest.begin(), rarest.end(),
              [](std::pair<uint8_t, size_t> const& a, std::pair<uint8_t, size_t> const& b) {
                  return a.second < b.second;
              });
    size_t const target = (n + count.size() - 1) / count.size();
    for (uint32_t node = 0; node < n; ++node) {
        if (count[col[node]] <= target) continue;
        for (size_t i = 0; i < rarest.size() && rarest[i].second < target; ++i) {
            uint8_t const nc = rarest[i].first;
            bool ok = true;
            for (uint32_t nb : s.nbr[node])
                if (col.at(nb) == nc) ok = false;
            if (!ok) continue;
            uint8_t const oc = col[node];
            --count[oc];
            ++count[nc];
            size_t iNew = 0, iOld = 0;
            for (size_t j = 0; j < rarest.size(); ++j) {
                if (rarest[j].first == oc) iOld = j;
                if (rarest[j].first == nc) iNew = j;
            }
            --rarest[iOld].second;
            ++rarest[iNew].second;
            // :279-283 bubble sort that swaps only on a strict '>' of the counts: it yields the
            // stable ascending order, which std::stable_sort reproduces exactly.
            std::stable_sort(rarest.begin(), rarest.end(),
                             [](std::pair<uint8_t, size_t> const& a, std::pair<uint8_t, size_t> const& b) {
                                 return a.second < b.second;
                             });
            col[node] = nc;
        }
    }
    return col;
}

// ---------------------------------------------------------------- sweep

struct Sorted {
    uint32_t nColors = 0;
    std::vector<uint32_t> groupStart;   // first sorted slot of each colour (no padding needed here)
    std::vector<uint32_t> groupSize;
    std::vector<uint32_t> newToOld;     // sorted slot -> original id
    std::vector<uint32_t> oldToNew;
};

// UpdaterGPUScBFM_AB_Type.cu:557-608: count per colour, then stable placement in original order.
Sorted group_by_colour(std::vector<uint8_t> const& col)
{
    Sorted g;
    uint32_t const n = (uint32_t)col.size();
    for (uint8_t c : col)
        if ((uint32_t)c + 1 > g.nColors) g.nColors = c + 1u;
    g.groupSize.assign(g.nColors, 0);
    for (uint8_t c : col) ++g.groupSize[c];
    g.groupStart.assign(g.nColors, 0);
    for (uint32_t c = 1; c < g.nColors; ++c) g.groupStart[c] = g.groupStart[c - 1] + g.groupSize[c - 1];
    std::vector<uint32_t> next = g.groupStart;
    g.newToOld.assign(n, 0);
    g.oldToNew.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const s = next[col[i]]++;
        g.oldToNew[i] = s;
        g.newToOld[s] = i;
    }
    return g;
}

struct Lattice {
    uint32_t mx, my, mz, lx, lxy;
    std::vector<uint8_t> cell;
    Lattice(uint32_t const* box)
        : mx(box[0] - 1), my(box[1] - 1), mz(box[2] - 1), lx(box[0]), lxy(box[0] * box[1]),
          cell((size_t)box[0] * box[1] * box[2], 0) {}
    inline size_t at(int32_t x, int32_t y, int32_t z) const
    {
        return (uint32_t(x) & mx) + (size_t)lx * (uint32_t(y) & my) + (size_t)lxy * (uint32_t(z) & mz);
    }
    // CRITICAL.cu:62-176 / :179-240: OR of the 3x3 plane at r0 + 2*d, +-1 in the two other axes.
    bool front_occupied(int32_t x, int32_t y, int32_t z, int dir) const
    {
        int const axis = dir >> 1;
        int const step = (dir & 1) ? 1 : -1;
        int32_t c[3] = {x, y, z};
        c[axis] += 2 * step;
        int const a1 = axis == 0 ? 1 : 0;
        int const a2 = axis == 2 ? 1 : 2;
        for (int u = -1; u <= 1; ++u)
            for (int v = -1; v <= 1; ++v) {
                int32_t p[3] = {c[0], c[1], c[2]};
                p[a1] += u;
                p[a2] += v;
                if (cell[at(p[0], p[1], p[2])]) return true;
            }
        return false;
    }
};

struct RunStats {
    uint64_t attempted = 0, tentative = 0, accepted = 0;
};

// DXTable/DYTable/DZTable, UpdaterGPUScBFM_AB_Type.cu:534-545: 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z
inline void dir_vec(int dir, int32_t& dx, int32_t& dy, int32_t& dz)
{
    int const s = (dir & 1) ? 1 : -1;
    dx = (dir >> 1) == 0 ? s : 0;
    dy = (dir >> 1) == 1 ? s : 0;
    dz = (dir >> 1) == 2 ? s : 0;
}

// Draw source: either the counter stream or an explicit list (2 words per sub-step).
struct Draws {
    int kind;               // 0 = counter, 1 = explicit
    uint64_t seed;
    uint64_t next;          // next draw index
    uint32_t const* list;
    uint64_t len;
    uint32_t get()
    {
        if (kind == 0) return counter_draw(seed, next++);
        if (next >= len) throw std::runtime_error("explicit draw list exhausted");
        return list[next++];
    }
};

// runSimulationOnGPU, CRITICAL.cu:501-573, with the kernels of CRITICAL.cu:298-411 run serially.
void sweep(System& s, Sorted const& g, Draws& draws, uint32_t nMcs, RunStats& st)
{
    uint32_t const n = s.n;
    // sorted copies (mPolymerSystemSorted, UpdaterGPUScBFM_AB_Type.cu:652-664)
    std::vector<int32_t> px(n), py(n), pz(n);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const k = g.oldToNew[i];
        px[k] = s.x[i]; py[k] = s.y[i]; pz[k] = s.z[i];
    }
    // neighbour ids re-indexed to sorted slots (:613-648)
    std::vector<std::vector<uint32_t>> nb(n);
    for (uint32_t i = 0; i < n; ++i) {
        auto& dst = nb[g.oldToNew[i]];
        for (uint32_t j : s.nbr[i]) dst.push_back(g.oldToNew[j]);
    }
    Lattice lat(s.lattice), tmp(s.lattice);
    for (uint32_t k = 0; k < n; ++k) lat.cell[lat.at(px[k], py[k], pz[k])] = 1;

    std::vector<uint8_t> flag(n, 0);
    for (uint32_t mcs = 0; mcs < nMcs; ++mcs) {
        for (uint32_t sub = 0; sub < g.nColors; ++sub) {
            uint32_t const c = draws.get() % g.nColors;
            uint32_t const seed = draws.get();
            uint32_t const off = g.groupStart[c], cnt = g.groupSize[c];
            st.attempted += cnt;
            // check, CRITICAL.cu:298-374
            for (uint32_t i = 0; i < cnt; ++i) {
                uint32_t const k = off + i;
                uint32_t const rn = move_hash(move_hash(i) ^ seed);
                int const dir = (int)(rn % 6u);
                int32_t dx, dy, dz;
                dir_vec(dir, dx, dy, dz);
                int32_t const x1 = px[k] + dx, y1 = py[k] + dy, z1 = pz[k] + dz;
                bool bad = outside_walls(s, x1, y1, z1);
                for (uint32_t j : nb[k]) {
                    if (bad) break;
                    if (s.forbidden[bond_index(px[j] - x1, py[j] - y1, pz[j] - z1)]) { bad = true; break; }
                }
                uint8_t f = 0;
                if (!bad && !lat.front_occupied(px[k], py[k], pz[k], dir)) {
                    f = (uint8_t)((dir << 2) | 1);
                    tmp.cell[tmp.at(x1, y1, z1)] = 1;
                    ++st.tentative;
                }
                flag[k] = f;
            }
            // perform + apply, CRITICAL.cu:376-411
            for (uint32_t i = 0; i < cnt; ++i) {
                uint32_t const k = off + i;
                if (!(flag[k] & 1)) continue;
                int const dir = (flag[k] >> 2) & 7;
                if (tmp.front_occupied(px[k], py[k], pz[k], dir)) continue;
                int32_t dx, dy, dz;
                dir_vec(dir, dx, dy, dz);
                lat.cell[lat.at(px[k], py[k], pz[k])] = 0;
                px[k] += dx; py[k] += dy; pz[k] += dz;
                lat.cell[lat.at(px[k], py[k], pz[k])] = 1;
                ++st.accepted;
            }
            // clear of the temporary lattice, CRITICAL.cu:561-573
            std::fill(tmp.cell.begin(), tmp.cell.end(), 0);
        }
    }
    // un-sort (CRITICAL.cu:686-695)
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const k = g.oldToNew[i];
        s.x[i] = px[k]; s.y[i] = py[k]; s.z[i] = pz[k];
    }
}

void set_err(char* err, int len, std::string const& msg)
{
    if (err && len > 0) {
        std::snprintf(err, (size_t)len, "%s", msg.c_str());
    }
}

System make_system(uint32_t n, int32_t const* xyz, uint32_t const* nbrCount, uint32_t const* nbrIds,
                   uint32_t maxc, uint32_t const* box, uint32_t walls, uint8_t const* forbidden)
{
    System s;
    s.n = n;
    s.walls = walls & 7u;
    for (int a = 0; a < 3; ++a) s.box[a] = box[a];
    s.x.resize(n); s.y.resize(n); s.z.resize(n);
    s.nbr.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        s.x[i] = xyz[3 * i]; s.y[i] = xyz[3 * i + 1]; s.z[i] = xyz[3 * i + 2];
        for (uint32_t j = 0; j < nbrCount[i]; ++j) {
            uint32_t const t = nbrIds[(size_t)i * maxc + j];
            if (t >= n) throw std::invalid_argument("neighbour id out of range");
            s.nbr[i].push_back(t);
        }
    }
    for (int i = 0; i < 512; ++i) s.forbidden[i] = forbidden[i] != 0;
    // The reference's lattice index needs power-of-two sides (UpdaterGPUScBFM_AB_Type.cu:797-848).
    // Generalised here to walled axes of any side >= 4: corners stay in [0, L-2] there, so the
    // axis never wraps and the box can sit in the lowest cells of a power-of-two side (the +-1
    // cells of a front plane at a wall then land on cells no corner occupies, as in the
    // reference's walled power-of-two boxes). Periodic axes still need a power of two.
    for (int a = 0; a < 3; ++a) {
        bool const p2 = box[a] != 0 && (box[a] & (box[a] - 1)) == 0;
        if (box[a] < 4 || (!((s.walls >> a) & 1u) && !p2))
            throw std::invalid_argument("box sides must be powers of two (any side >= 4 along a walled axis)");
        uint32_t P = 4;
        while (P < box[a]) P *= 2;
        s.lattice[a] = P;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (outside_walls(s, s.x[i], s.y[i], s.z[i]))
            throw std::invalid_argument("monomer " + std::to_string(i) + " lies outside the walls of the box");
    return s;
}

// ---------------------------------------------------------------- CPU baseline
//
// Random-sequential single-monomer BFM update (the LeMonADE serial-updater scheme, which is not
// in the reference tree): each attempt picks a random monomer and one of the 6 unit moves, applies
// the same bond-set and excluded-volume rules, and moves it at once. N attempts per MCS.
// xoshiro128** (Blackman & Vigna 2018) supplies the picks.
struct Xoshiro128 {
    uint32_t s[4];
    explicit Xoshiro128(uint64_t seed)
    {
        uint64_t z = seed;
        for (int i = 0; i < 4; ++i) { z = sm64_mix(z + 0x9E3779B97F4A7C15ull * (i + 1)); s[i] = (uint32_t)(z >> 32); }
        if (!(s[0] | s[1] | s[2] | s[3])) s[0] = 1;
    }
    static inline uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
    inline uint32_t next()
    {
        uint32_t const r = rotl(s[1] * 5u, 7) * 9u;
        uint32_t const t = s[1] << 9;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 11);
        return r;
    }
};

void sequential_sweep(System& s, uint64_t seed, uint32_t nMcs, RunStats& st)
{
    Lattice lat(s.lattice);
    for (uint32_t k = 0; k < s.n; ++k) lat.cell[lat.at(s.x[k], s.y[k], s.z[k])] = 1;
    Xoshiro128 rng(seed);
    uint64_t const attempts = (uint64_t)nMcs * s.n;
    for (uint64_t a = 0; a < attempts; ++a) {
        uint32_t const r = rng.next();
        uint32_t const k = (uint32_t)(((uint64_t)r * s.n) >> 32);
        int const dir = (int)(rng.next() % 6u);
        int32_t dx, dy, dz;
        dir_vec(dir, dx, dy, dz);
        int32_t const x1 = s.x[k] + dx, y1 = s.y[k] + dy, z1 = s.z[k] + dz;
        bool bad = outside_walls(s, x1, y1, z1);
        for (uint32_t j : s.nbr[k])
            if (!bad && s.forbidden[bond_index(s.x[j] - x1, s.y[j] - y1, s.z[j] - z1)]) { bad = true; break; }
        ++st.attempted;
        if (bad || lat.front_occupied(s.x[k], s.y[k], s.z[k], dir)) continue;
        lat.cell[lat.at(s.x[k], s.y[k], s.z[k])] = 0;
        s.x[k] = x1; s.y[k] = y1; s.z[k] = z1;
        lat.cell[lat.at(x1, y1, z1)] = 1;
        ++st.accepted;
    }
}

}  // namespace

// ====================================================================== C ABI (ctypes)
extern "C" {

uint32_t orc_hash(uint32_t a) { return move_hash(a); }

uint32_t orc_counter_draw(uint64_t seed, uint64_t k) { return counter_draw(seed, k); }

// Fills `out` with `count` draws of the counter stream starting at draw index k0.
void orc_counter_draws(uint64_t seed, uint64_t k0, uint64_t count, uint32_t* out)
{
    for (uint64_t i = 0; i < count; ++i) out[i] = counter_draw(seed, k0 + i);
}

uint32_t orc_bond_index(int32_t dx, int32_t dy, int32_t dz) { return bond_index(dx, dy, dz); }

// Colours the bond graph exactly as graphColoring.tpp does. Returns the colour count, or -1.
int orc_color(uint32_t n, uint32_t const* nbrCount, uint32_t const* nbrIds, uint32_t maxc,
              uint8_t* colorsOut, char* err, int errLen)
{
    try {
        if (n == 0) throw std::invalid_argument("no monomers");
        System s;
        s.n = n;
        s.nbr.resize(n);
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = 0; j < nbrCount[i]; ++j) {
                uint32_t const t = nbrIds[(size_t)i * maxc + j];
                if (t >= n) throw std::invalid_argument("neighbour id out of range");
                s.nbr[i].push_back(t);
            }
        std::vector<uint8_t> const col = colour_graph(s);
        int nc = 0;
        for (uint32_t i = 0; i < n; ++i) {
            colorsOut[i] = col[i];
            if (col[i] + 1 > nc) nc = col[i] + 1;
        }
        return nc;
    } catch (std::exception const& e) {
        set_err(err, errLen, e.what());
        return -1;
    }
}

// Runs nMcs Monte Carlo steps of the parallel (colour-by-colour) sweep.
//   drawKind 0: counter stream (seed, starting draw index = 2*subStep0)
//   drawKind 1: explicit draws list (2 per sub-step), consumed from index 0
// stats[0..2] += attempted, tentatively accepted, accepted.
int orc_run(uint32_t n, int32_t const* xyzIn, uint32_t const* nbrCount, uint32_t const* nbrIds,
            uint32_t maxc, uint32_t const* box, uint32_t walls, uint8_t const* forbidden, int drawKind, uint64_t seed,
            uint64_t subStep0, uint32_t const* drawList, uint64_t drawLen, uint32_t nMcs,
            int32_t* xyzOut, uint64_t* stats, char* err, int errLen)
{
    try {
        if (n == 0) throw std::invalid_argument("no monomers");
        System s = make_system(n, xyzIn, nbrCount, nbrIds, maxc, box, walls, forbidden);
        uint32_t nAllowed = 0;
        for (int i = 0; i < 512; ++i) nAllowed += s.forbidden[i] ? 0 : 1;
        if (nAllowed != 108)   // UpdaterGPUScBFM_AB_Type.cu:521-528
            throw std::runtime_error("Wrong bond-set! Expected 108 allowed bonds, but got " + std::to_string(nAllowed));
        std::vector<uint8_t> const col = colour_graph(s);
        Sorted const g = group_by_colour(col);
        Draws d{drawKind, seed, drawKind == 0 ? 2 * subStep0 : 0, drawList, drawLen};
        RunStats st;
        sweep(s, g, d, nMcs, st);
        for (uint32_t i = 0; i < n; ++i) {
            xyzOut[3 * i] = s.x[i]; xyzOut[3 * i + 1] = s.y[i]; xyzOut[3 * i + 2] = s.z[i];
        }
        if (stats) { stats[0] += st.attempted; stats[1] += st.tentative; stats[2] += st.accepted; }
        return 0;
    } catch (std::exception const& e) {
        set_err(err, errLen, e.what());
        return -1;
    }
}

// Random-sequential CPU baseline; stats[0..1] += attempted, accepted.
int orc_seq_run(uint32_t n, int32_t const* xyzIn, uint32_t const* nbrCount, uint32_t const* nbrIds,
                uint32_t maxc, uint32_t const* box, uint32_t walls, uint8_t const* forbidden, uint64_t seed, uint32_t nMcs,
                int32_t* xyzOut, uint64_t* stats, char* err, int errLen)
{
    try {
        System s = make_system(n, xyzIn, nbrCount, nbrIds, maxc, box, walls, forbidden);
        RunStats st;
        sequential_sweep(s, seed, nMcs, st);
        for (uint32_t i = 0; i < n; ++i) {
            xyzOut[3 * i] = s.x[i]; xyzOut[3 * i + 1] = s.y[i]; xyzOut[3 * i + 2] = s.z[i];
        }
        if (stats) { stats[0] += st.attempted; stats[1] += st.accepted; }
        return 0;
    } catch (std::exception const& e) {
        set_err(err, errLen, e.what());
        return -1;
    }
}

}  // extern "C"
