/*
 * bfm_host.hpp -- host-side algorithms that fix the trajectory of the colored
 * sweep: the R250 colour/seed generator and the species (graph) colouring.
 *
 * Both must give the same numbers as the reference's host code for the GPU
 * kernels to reproduce its trajectories bit for bit.
 */
#pragma once
#include <algorithm>
#include <cstdint>
#include <stack>
#include <stdexcept>
#include <utility>
#include <vector>

namespace bfm {

/* R250 shift-register generator (Kirkpatrick & Stoll 1981, buffer set-up
 * after W. L. Maier 1991): x[n] = x[n-250] ^ x[n-147], the partner word 103
 * slots ahead in the 250-word ring.  Stands in for
 * LeMonADE's RandomNumberGenerators::r250_rand32, which the reference calls
 * twice per colour substep (UpdaterGPUScBFM_AB_Type.cu:3065-3066). */
struct R250 {
    uint32_t buf[250];
    uint32_t idx = 0;

    void seed_words(const uint32_t *w)
    {
        for (int k = 0; k < 250; ++k) buf[k] = w[k];
        for (int j = 0; j < 32; ++j) {
            const int k = 7 * j + 3;
            buf[k] = (buf[k] & (0xFFFFFFFFu >> j)) | (0x80000000u >> j);
        }
        idx = 0;
    }
    void seed_u64(uint64_t s)
    {
        uint32_t w[250];
        for (int k = 0; k < 250; ++k) {
            uint64_t z = (s += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            w[k] = (uint32_t)((z ^ (z >> 31)) >> 32);
        }
        seed_words(w);
    }
    uint32_t next()
    {
        const uint32_t i = idx;
        const uint32_t j = i >= 147u ? i - 147u : i + 103u;
        buf[i] ^= buf[j];
        idx = i >= 249u ? 0u : i + 1u;
        return buf[i];
    }
};

/* Species colouring of the bond graph, the reference's graphColoring()
 * (graphColoring.tpp:103-439) with bUniformColors = true
 * (UpdaterGPUScBFM_AB_Type.cu:1565):
 *  1. walk each connected component depth-first from its lowest id, give
 *     every node the smallest colour none of its coloured neighbours has,
 *     continue at the first uncoloured neighbour and remember nodes with more
 *     than one uncoloured neighbour on a stack;
 *  2. rebalance: in id order, a node whose colour holds more than
 *     ceil(n / nColours) nodes is moved to the rarest colour its neighbours
 *     do not use, scanning the colours rarest-first (the scan goes on after a
 *     move, as in the reference).
 * nbr holds 8 slots per node.  Throws std::runtime_error past 255 colours. */
/* The walk of step 1 over the nodes whose colour is still kNoColor (whole
 * components: a component is either coloured already or not at all), in
 * the reference's order; count receives every colour's node count. */
constexpr uint32_t kNoColor = 0xFFFFFFFFu;
inline void dfs_colors_rest(uint32_t n, const uint8_t *deg, const uint32_t *nbr, std::vector<uint32_t> &color,
                            std::vector<size_t> &count)
{
    const uint32_t kNone = kNoColor;
    const int64_t kNoNode = -1;
    count.clear();
    for (uint32_t i = 0; i < n; ++i)
        if (color[i] != kNone) {
            if (color[i] >= count.size()) count.resize(color[i] + 1, 0);
            ++count[color[i]];
        }
    std::vector<uint8_t> taken(256);
    for (uint32_t root = 0; root < n; ++root) {
        if (color[root] != kNone) continue;
        std::stack<uint32_t> branch;
        int64_t cur = root;
        for (;;) {
            std::fill(taken.begin(), taken.end(), 0);
            uint32_t open = 0;
            int64_t next = kNoNode;
            for (uint32_t j = 0; j < deg[cur]; ++j) {
                const uint32_t v = nbr[(size_t)cur * 8 + j];
                if (color[v] != kNone) taken[color[v]] = 1;
                else if (open++ == 0) next = v;
            }
            uint32_t c = 0;
            while (c < 255 && taken[c]) ++c;
            if (c == 255)
                throw std::runtime_error("Already used up the maximum amount of colors. Can't color the given polymer system automatically!");
            color[cur] = c;
            if (c >= count.size()) count.resize(c + 1, 0);
            ++count[c];
            if (open == 0 && branch.empty()) break;
            if (open > 1) branch.push((uint32_t)cur);
            cur = next;
            if (open == 0) {
                while (!branch.empty()) {
                    cur = branch.top();
                    uint32_t open2 = 0;
                    int64_t next2 = kNoNode;
                    for (uint32_t j = 0; j < deg[cur]; ++j) {
                        const uint32_t v = nbr[(size_t)cur * 8 + j];
                        if (color[v] == kNone && open2++ == 0) next2 = v;
                    }
                    if (open2 < 2) branch.pop();
                    if (next2 != kNoNode) {
                        cur = next2;
                        break;
                    }
                    cur = kNoNode;
                }
                if (branch.empty() && cur == kNoNode) break;
            }
        }
    }
}

inline std::vector<uint32_t> dfs_colors(uint32_t n, const uint8_t *deg, const uint32_t *nbr, std::vector<size_t> &count)
{
    std::vector<uint32_t> color(n, kNoColor);
    dfs_colors_rest(n, deg, nbr, color, count);
    return color;
}

/* step 2 of color_graph on a colouring and its colour counts */
inline void rebalance_colors(uint32_t n, const uint8_t *deg, const uint32_t *nbr, std::vector<uint32_t> &color,
                             std::vector<size_t> &count)
{
    if (!count.empty()) {
        using Entry = std::pair<uint32_t, size_t>;
        const size_t k = count.size();
        std::vector<Entry> rarest(k);
        for (size_t i = 0; i < k; ++i) rarest[i] = Entry((uint32_t)i, count[i]);
        auto by_count = [](const Entry &a, const Entry &b) { return a.second < b.second; };
        std::sort(rarest.begin(), rarest.end(), by_count);
        const size_t limit = ((size_t)n + k - 1) / k;
        for (uint32_t v = 0; v < n; ++v) {
            if (count[color[v]] <= limit) continue;
            for (size_t i = 0; i < k && rarest[i].second < limit; ++i) {
                const uint32_t to = rarest[i].first;
                bool free_ = true;
                for (uint32_t j = 0; j < deg[v]; ++j)
                    if (color[nbr[(size_t)v * 8 + j]] == to) free_ = false;
                if (!free_) continue;
                const uint32_t from = color[v];
                --count[from];
                ++count[to];
                for (auto &e : rarest) {
                    if (e.first == from) --e.second;
                    if (e.first == to) ++e.second;
                }
                std::stable_sort(rarest.begin(), rarest.end(), by_count);
                color[v] = to;
            }
        }
    }
}

inline std::vector<uint32_t> color_graph(uint32_t n, const uint8_t *deg, const uint32_t *nbr, bool uniform)
{
    std::vector<size_t> count;
    std::vector<uint32_t> color = dfs_colors(n, deg, nbr, count);
    if (uniform) rebalance_colors(n, deg, nbr, color, count);
    return color;
}

} // namespace bfm
