/*
 * oracle/ref_host.cpp -- TEST INFRASTRUCTURE.
 *
 * Exposes the reference's own host-compilable pieces through a C ABI so the
 * CPU restatement in oracle/bfm_oracle.cpp (and the golden fixtures in
 * tests/golden/) can be pinned against them:
 *   rngs/Saru.h   (Rngs::Saru, used by the check kernel, .cu:957-965)
 *   rngs/Hash.h   (Rngs::Hash, the reference's default RNG, .cu:1407)
 *   graphColoring.tpp (the species colouring, called at .cu:1566-1570)
 * Built by oracle/Makefile from the sources under the reference tree into
 * oracle/_ref/libref_host.so.
 */
#include <vector_types.h>   /* uint2, used by Rngs::Saru */
#include <cstdint>
#include <cstddef>
#include <vector>
#include <stdexcept>

#include "rngs/Saru.h"
#include "rngs/Hash.h"
#include "graphColoring.tpp"

namespace {
struct Edges {
    uint32_t size;
    uint32_t ids[8];
};
}

extern "C" {

uint32_t ref_saru(uint32_t seed, uint64_t iteration, uint32_t subseq)
{
    Rngs::Saru r;
    r.setSeed(seed);
    r.setIteration(iteration);
    r.setSubsequence(subseq);
    return r.rng32();
}

uint32_t ref_hash(uint32_t seed, uint32_t subseq)
{
    Rngs::Hash r;
    r.setSeed(seed);
    r.setSubsequence(subseq);
    return r.rng32();
}

/* same call as UpdaterGPUScBFM_AB_Type.cu:1566-1570 (T_Id = T_Color = uint32_t) */
int ref_graph_coloring(uint32_t n, const uint32_t *nnbr, const uint32_t *nbr8, int uniform, uint32_t *out)
{
    std::vector<Edges> e(n);
    for (uint32_t i = 0; i < n; ++i) {
        e[i].size = nnbr[i];
        for (uint32_t j = 0; j < 8; ++j) e[i].ids[j] = nbr8[(size_t)i * 8 + j];
    }
    Edges const *p = e.data();
    try {
        auto c = graphColoring<Edges const *, uint32_t, uint32_t>(
            p, n, uniform != 0, [](Edges const *const &x, uint32_t const &i) { return (size_t)x[i].size; },
            [](Edges const *const &x, uint32_t const &i, size_t const &j) { return x[i].ids[j]; });
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            out[i] = c[i];
            if (c[i] + 1 > k) k = c[i] + 1;
        }
        return (int)k;
    } catch (...) {
        return -1;
    }
}

} /* extern "C" */
