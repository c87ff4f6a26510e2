/*
 * oracle/r250.h -- TEST INFRASTRUCTURE (oracle side). Not part of the product.
 *
 * The host random number generator that drives the colour and seed draws of
 * the colored BFM sweep.  The reference draws them with LeMonADE's
 * RandomNumberGenerators::r250_rand32() (UpdaterGPUScBFM_AB_Type.cu:3065-3066,
 * member declared at UpdaterGPUScBFM_AB_Type.h:230).  LeMonADE is an
 * un-vendored submodule (.gitmodules:1-3, no pinned commit), so this file
 * restates the published R250 shift-register generator:
 *
 *   Kirkpatrick & Stoll, J. Comput. Phys. 40 (1981) 517:
 *       x[n] = x[n-250] XOR x[n-147]   (the partner word sits 103 slots
 *       ahead in the 250-word ring; reciprocal of x^250 + x^103 + 1)
 *   buffer set-up as in W. L. Maier, Dr. Dobb's Journal (May 1991):
 *       250 seed words, then a triangular bit pattern on the words
 *       k = 7*j + 3 (j = 0..31) so that the 32 bit-columns are independent.
 *
 * The same definition is used by the oracle, by the shim header that lets the
 * reference's own updater build (oracle/ref_shim), and -- in an independent
 * copy -- by the product.  Parity against LeMonADE's own R250 / .seeds
 * reader is UNPINNED (its source is absent).
 */
#pragma once
#include <cstdint>

namespace orc {

struct R250State {
    uint32_t buf[250];
    uint32_t idx;
};

inline void r250_seed_words(R250State &s, const uint32_t *w)
{
    for (int k = 0; k < 250; ++k) s.buf[k] = w[k];
    for (int j = 0; j < 32; ++j) {
        const int k = 7 * j + 3;
        s.buf[k] &= (0xFFFFFFFFu >> j);
        s.buf[k] |= (0x80000000u >> j);
    }
    s.idx = 0;
}

/* splitmix64 (Steele, Lea & Flood 2014) expands one 64-bit seed into words */
inline uint64_t splitmix64_next(uint64_t &x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline void r250_seed_u64(R250State &s, uint64_t seed)
{
    uint32_t w[250];
    uint64_t x = seed;
    for (int k = 0; k < 250; ++k) w[k] = (uint32_t)(splitmix64_next(x) >> 32);
    r250_seed_words(s, w);
}

inline uint32_t r250_next(R250State &s)
{
    const uint32_t i = s.idx;
    const uint32_t j = (i >= 147u) ? i - 147u : i + 103u;
    const uint32_t v = (s.buf[i] ^= s.buf[j]);
    s.idx = (i >= 249u) ? 0u : i + 1u;
    return v;
}

} // namespace orc
