// Graph colouring of the bond graph, with the reference's exact results.
//
// Behaviour of src/pscbfm/graphColoring.tpp:77-293 called with bUniformColors = true
// (src/pscbfm/UpdaterGPUScBFM_AB_Type.cu:550-555):
//  1. Nodes are visited in id order; an uncoloured node starts a depth-first walk of its molecule
//     (:97-212). Each visited node takes the smallest colour not used by an already coloured
//     listed neighbour (:142-153); the walk continues at the first uncoloured listed neighbour
//     and backtracks through a stack of nodes that had more than one uncoloured neighbour.
//  2. Uniform pass (:216-290): colours sorted rarest first by an unstable std::sort; every node of
//     an over-full colour tries the under-full colours in that order and takes each one that no
//     listed neighbour has, re-sorting the (stable) order after every change.
// Colour IDs and the in-colour order derived from them select the random direction of every
// move, so the result must be identical, including the tie-breaking of the std::sort.

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "bfm_engine.hpp"

namespace bfm {

std::vector<uint8_t> colour_bond_graph(uint32_t n, uint32_t const* cnt, uint32_t const* ids, uint32_t stride)
{
    constexpr uint8_t kUncoloured = 255;
    constexpr uint32_t kColourLimit = 255;
    std::vector<uint8_t> colour(n, kUncoloured);
    std::vector<size_t> freq;
    // generation-stamped "colour seen among neighbours" marks, so nothing is cleared per node
    std::vector<uint32_t> seen(256, 0);
    uint32_t gen = 0;

    auto nbrs = [&](uint32_t v) { return std::make_pair(ids + (size_t)v * stride, ids + (size_t)v * stride + cnt[v]); };

    auto uncoloured_scan = [&](uint32_t v, uint32_t& first) {
        uint32_t count = 0;
        first = UINT32_MAX;
        auto r = nbrs(v);
        for (auto p = r.first; p != r.second; ++p)
            if (colour[*p] == kUncoloured) {
                if (count++ == 0) first = *p;
            }
        return count;
    };

    auto assign = [&](uint32_t v) {
        ++gen;
        auto r = nbrs(v);
        for (auto p = r.first; p != r.second; ++p)
            if (colour[*p] != kUncoloured) seen[colour[*p]] = gen;
        uint32_t c = 0;
        while (c < kColourLimit && seen[c] == gen) ++c;
        if (c == kColourLimit)
            throw std::runtime_error(
                "Already used up the maximum amount of colors. Can't color the given polymer system automatically!");
        colour[v] = (uint8_t)c;
        if (c >= freq.size()) freq.resize(c + 1, 0);
        ++freq[c];
    };

    std::vector<uint32_t> stack;
    for (uint32_t root = 0; root < n; ++root) {
        if (colour[root] != kUncoloured) continue;
        stack.clear();
        uint32_t v = root;
        bool walking = true;
        while (walking) {
            uint32_t next;
            uint32_t const open = uncoloured_scan(v, next);
            assign(v);
            if (open == 0 && stack.empty()) break;
            if (open > 1) stack.push_back(v);
            if (open > 0) {
                v = next;
                continue;
            }
            // dead end: resume from the most recent branching node that still has work
            walking = false;
            while (!stack.empty()) {
                uint32_t const b = stack.back();
                uint32_t nb;
                uint32_t const left = uncoloured_scan(b, nb);
                if (left < 2) stack.pop_back();
                if (left > 0) {
                    v = nb;
                    walking = true;
                    break;
                }
            }
        }
    }

    // uniform pass
    using Entry = std::pair<uint8_t, size_t>;
    std::vector<Entry> order(freq.size());
    for (size_t c = 0; c < freq.size(); ++c) order[c] = Entry((uint8_t)c, freq[c]);
    auto byCount = [](Entry const& a, Entry const& b) { return a.second < b.second; };
    std::sort(order.begin(), order.end(), byCount);
    size_t const target = (n + freq.size() - 1) / freq.size();
    for (uint32_t v = 0; v < n; ++v) {
        if (freq[colour[v]] <= target) continue;
        for (size_t i = 0; i < order.size() && order[i].second < target; ++i) {
            uint8_t const cand = order[i].first;
            bool clash = false;
            auto r = nbrs(v);
            for (auto p = r.first; p != r.second; ++p) clash = clash || colour[*p] == cand;
            if (clash) continue;
            uint8_t const old = colour[v];
            --freq[old];
            ++freq[cand];
            for (auto& e : order) {
                if (e.first == old) --e.second;
                if (e.first == cand) ++e.second;
            }
            std::stable_sort(order.begin(), order.end(), byCount);
            colour[v] = cand;
        }
    }
    return colour;
}

}  // namespace bfm
