/*
 * oracle/bfm_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the reference's colored bond-fluctuation-model sweep
 * (lgh0504/pscbfm, src/pscbfm/UpdaterGPUScBFM_AB_Type.cu).  It is the checker
 * for the product's CUDA path: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg / reference arm of bench.py load it.  The product never
 * links it and never falls back to it.
 *
 * Parity pins:
 *   - RNG kernels (Saru, Hash) and the graph colouring are compared in CPU
 *     tests against the reference's own headers (rngs/Saru.h, rngs/Hash.h,
 *     graphColoring.tpp) compiled from its sources into oracle/_ref/.
 *   - The whole sweep is compared on the GPU against the reference's own
 *     updater (UpdaterGPUScBFM_AB_Type.cu built for sm_100a, oracle/_ref/).
 *   - The host R250 generator of LeMonADE is absent from the reference tree;
 *     oracle/r250.h restates the published R250 and that one part is unpinned.
 *
 * Every function below cites the reference lines it restates.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stack>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include <atomic>
#include <omp.h>

#include "r250.h"

namespace orc {

/* ------------------------------------------------------------------ RNGs */

/* Saru (S. Worley, HOOMD-blue): seed premix + one LCG/Weyl step.
 * Restates rngs/Saru.h:153-170 (init), :240-247 (u32<1>), :257-261 (Weyl<1>).
 * The caller passes (seed, iteration, subsequence) already truncated to
 * 32 bits, as Saru::rng32 does (Saru.h:35-40). */
static inline uint32_t saru_u32(uint32_t s1, uint32_t s2, uint32_t s3)
{
    s3 ^= (s1 << 7) ^ (s2 >> 6);
    s2 += (s1 >> 4) ^ (s3 >> 15);
    s1 ^= (s2 << 9) + (s3 << 8);
    s3 ^= 0xA5366B4Du * ((s2 >> 11) ^ (s1 << 1));
    s2 += 0x72BE1579u * ((s1 << 4) ^ (s3 >> 16));
    s1 ^= 0x3F38A6EDu * ((s3 >> 5) ^ (uint32_t)((int32_t)s2 >> 22));
    s2 += s1 * s3;
    s1 += s3 ^ (s2 >> 2);
    s2 ^= (uint32_t)((int32_t)s2 >> 17);
    uint32_t lcg = 0x79DEDEA3u * (s1 ^ (uint32_t)((int32_t)s1 >> 14));
    uint32_t weyl = (lcg + s2) ^ (uint32_t)((int32_t)lcg >> 8);
    lcg = lcg + weyl * (weyl ^ 0xDDDF97F5u);
    weyl = 0xABCB96F7u + (weyl >> 1);
    lcg = 0x4BEB5D59u * lcg + 0x2600E1F7u;
    weyl = weyl + 0x8009D14Bu + ((uint32_t)((int32_t)weyl >> 31) & 0xDA879ADDu);
    const uint32_t v = (lcg ^ (lcg >> 26)) + weyl;
    return (v ^ (v >> 20)) * 0x6957F5A7u;
}

/* Robert Jenkins' 32-bit integer hash, as used by rngs/Hash.h:24-46 */
static inline uint32_t jenkins_hash(uint32_t a)
{
    a = (a + 0x7ED55D16u) + (a << 12);
    a = (a ^ 0xC761C23Cu) ^ (a >> 19);
    a = (a + 0x165667B1u) + (a << 5);
    a = (a + 0xD3A2646Cu) ^ (a << 9);
    a = (a + 0xFD7046C5u) + (a << 3);
    a = (a ^ 0xB55A4F09u) ^ (a >> 16);
    return a;
}

/* Hash::rng32 (Hash.h:65-69): state = subsequence, hash(hash(state) ^ seed) */
static inline uint32_t hash_rng(uint32_t seed, uint32_t subseq)
{
    return jenkins_hash(jenkins_hash(subseq) ^ seed);
}

enum { RNG_INTHASH = 1, RNG_SARU = 2, RNG_PHILOX = 3 };

/* Philox4x32-10 (Salmon et al., SC'11, the Random123 constants), the word
 * curand() returns after curand_init(seed, subsequence, offset) -- the use
 * in rngs/lemonade_philox.h:48-56: block counter (offset/4) + subsequence *
 * 2^64, key = seed, word offset % 4.  Pinned against curand on the GPU. */
static inline uint32_t philox4x32_10(uint64_t seed, uint64_t subsequence, uint64_t offset)
{
    const uint64_t blk = offset >> 2;
    uint32_t c[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)subsequence, (uint32_t)(subsequence >> 32)};
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = (uint32_t)p1;
        c[2] = n2;
        c[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c[offset & 3];
}

/* ---------------------------------------------------------- Z-order index */

/* 10-bit -> 30-bit dilation with two zero bits between payload bits.  Equal to
 * diluteBits<uint32_t,2> (UpdaterGPUScBFM_AB_Type.cu:204-230) for inputs
 * below 1024. */
static inline uint32_t dilate3(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

/* linearizeBoxVectorIndex with USE_ZCURVE_FOR_LATTICE (.cu:289-316) */
static inline uint32_t zindex(int64_t x, int64_t y, int64_t z, uint32_t mx, uint32_t my, uint32_t mz)
{
    return dilate3((uint32_t)x & mx) | (dilate3((uint32_t)y & my) << 1) | (dilate3((uint32_t)z & mz) << 2);
}

/* linearizeBondVectorIndex (.cu:871-889) */
static inline uint32_t bond_index(int64_t dx, int64_t dy, int64_t dz)
{
    return (uint32_t)(dx & 7) | ((uint32_t)(dy & 7) << 3) | ((uint32_t)(dz & 7) << 6);
}

/* ------------------------------------------------------- graph colouring */

/* Restates graphColoring() (graphColoring.tpp:103-439): a depth-first greedy
 * colouring (smallest colour not used by an already coloured neighbour, walk
 * to the first uncoloured neighbour, stack the node when it has more than one
 * uncoloured neighbour), optionally followed by the uniform rebalancing pass
 * (:323-418) which moves nodes of over-full colours to the rarest colour that
 * none of their neighbours has.  The rarest-first list is ordered with the
 * same std::sort call as the reference (:335-338) and re-ordered after each
 * change by a stable sort on the frequency (:390-394 use a stable bubble sort). */
static std::vector<uint32_t> graph_coloring(uint32_t n, const uint32_t *nnbr, const uint32_t *nbr, bool uniform)
{
    const uint32_t NONE = 0xFFFFFFFFu;
    const long long cNoNode = -1;
    const uint32_t nMaxColors = 255;
    std::vector<uint32_t> color(n, NONE);
    std::vector<size_t> freq;
    std::vector<uint8_t> used;
    for (uint32_t start = 0; start < n; ++start) {
        if (color[start] != NONE) continue;
        std::stack<uint32_t> todo;
        long long node = start;
        while (true) {
            used.assign(257, 0);
            size_t nUncolored = 0;
            long long firstUncolored = cNoNode;
            for (uint32_t j = 0; j < nnbr[node]; ++j) {
                const uint32_t nb = nbr[(size_t)node * 8 + j];
                const uint32_t c = color[nb];
                if (c != NONE) used[c] = 1;
                else {
                    ++nUncolored;
                    if (firstUncolored == cNoNode) firstUncolored = nb;
                }
            }
            uint32_t c = 0;
            while (c < nMaxColors && used[c]) ++c;
            if (c == nMaxColors)
                throw std::runtime_error("Already used up the maximum amount of colors. Can't color the given polymer system automatically!");
            color[node] = c;
            if (c >= freq.size()) freq.resize(c + 1, 0);
            ++freq[c];
            if (nUncolored == 0 && todo.empty()) break;
            if (nUncolored > 1) todo.push((uint32_t)node);
            node = firstUncolored;
            if (nUncolored == 0) {
                while (!todo.empty()) {
                    node = todo.top();
                    size_t n2 = 0;
                    long long first2 = cNoNode;
                    for (uint32_t j = 0; j < nnbr[node]; ++j) {
                        const uint32_t nb = nbr[(size_t)node * 8 + j];
                        if (color[nb] == NONE) {
                            ++n2;
                            if (first2 == cNoNode) first2 = nb;
                        }
                    }
                    if (n2 < 2) todo.pop();
                    if (first2 != cNoNode) { node = first2; break; }
                    node = cNoNode;
                }
                if (todo.empty() && node == cNoNode) break;
            }
        }
    }
    if (uniform && !freq.empty()) {
        const size_t k = freq.size();
        std::vector<std::pair<uint32_t, size_t>> rare(k);
        for (size_t i = 0; i < k; ++i) rare[i] = {(uint32_t)i, freq[i]};
        std::sort(rare.begin(), rare.end(),
                  [](const std::pair<uint32_t, size_t> &a, const std::pair<uint32_t, size_t> &b) { return a.second < b.second; });
        const size_t target = ((size_t)n + k - 1) / k;
        for (uint32_t node = 0; node < n; ++node) {
            if (freq[color[node]] <= target) continue;
            for (size_t i = 0; i < k && rare[i].second < target; ++i) {
                const uint32_t nc = rare[i].first;
                bool ok = true;
                for (uint32_t j = 0; j < nnbr[node]; ++j)
                    if (color[nbr[(size_t)node * 8 + j]] == nc) ok = false;
                if (!ok) continue;
                const uint32_t oc = color[node];
                --freq[oc];
                ++freq[nc];
                size_t iNew = 0, iOld = 0;
                for (size_t q = 0; q < k; ++q) {
                    if (rare[q].first == oc) iOld = q;
                    if (rare[q].first == nc) iNew = q;
                }
                --rare[iOld].second;
                ++rare[iNew].second;
                std::stable_sort(rare.begin(), rare.end(),
                                 [](const std::pair<uint32_t, size_t> &a, const std::pair<uint32_t, size_t> &b) { return a.second < b.second; });
                color[node] = nc;
            }
        }
    }
    return color;
}

/* ------------------------------------------------- colored sweep emulator */

static const int DX[6] = {-1, 1, 0, 0, 0, 0};
static const int DY[6] = {0, 0, -1, 1, 0, 0};
static const int DZ[6] = {0, 0, 0, 0, -1, 1};

struct Sweep {
    uint32_t Lx = 0, Ly = 0, Lz = 0, mx = 0, my = 0, mz = 0;
    uint32_t n = 0;
    std::vector<uint32_t> nnbr, nbr;          /* nbr: n x 8, original ids */
    uint8_t forbidden[512];
    int rng = RNG_SARU;
    int64_t age = 0;
    int64_t sortEvery = 5000;
    std::vector<int64_t> px, py, pz;          /* absolute positions */
    std::vector<uint32_t> color;
    uint32_t nSpecies = 0;
    std::vector<std::vector<uint32_t>> slab;  /* slab[s][i] = original id */
    std::vector<uint8_t> lattice, tmp;
    std::vector<uint8_t> flags;
    std::vector<uint32_t> target;
    uint64_t nAttempt = 0, nCandidate = 0, nAccept = 0;
    int nThreads = 1;
    bool periodic[3] = {true, true, true};
    /* filter statistics of the reference's "Stats" mode (.cu:2917-2936):
     * per species and filter, over the substeps of the latest run */
    int filterStats = 0; /* 0 off, 1 counted as the reference's count kernels, 2 the moves made */
    std::vector<double> fsum, fsum2, fmin, fmax, fcnt;

    /* the box test of the check kernel for non-periodic axes (.cu:988-996),
     * on the reference's unsigned device coordinates (a step below 0 wraps
     * to the type's maximum), with the axis' own box size */
    bool inside(int64_t c0, int64_t c1, int64_t L) const
    {
        if (c1 < 0) return false;
        return (0 < c0 && c1 < L - 1) || (c0 == 0 && c1 <= 1) || (c0 == L - 1 && c1 > 1);
    }

    /* lattice index: Z-order of the wrapped coordinates in the box padded to
     * powers of two (masking is the wrap when the edges are powers of two,
     * as in the reference; edges that are only multiples of 8 wrap mod L) */
    bool pow2 = true;
    static int64_t wrap(int64_t v, int64_t L)
    {
        const int64_t r = v % L;
        return r < 0 ? r + L : r;
    }
    uint32_t z(int64_t x, int64_t y, int64_t zz) const
    {
        if (pow2) return zindex(x, y, zz, mx, my, mz);
        return zindex(wrap(x, Lx), wrap(y, Ly), wrap(zz, Lz), mx, my, mz);
    }

    /* doSpatialSorting (.cu:1835-1943): per species, order by the Z-curve
     * index of the wrapped position.  The keys are unique (excluded volume),
     * so any correct sort gives the reference's order. */
    void spatialSort()
    {
        for (auto &s : slab) {
            std::vector<std::pair<uint32_t, uint32_t>> kv(s.size());
            for (size_t i = 0; i < s.size(); ++i) kv[i] = {z(px[s[i]], py[s[i]], pz[s[i]]), s[i]};
            std::sort(kv.begin(), kv.end());
            for (size_t i = 0; i < s.size(); ++i) s[i] = kv[i].second;
        }
    }

    /* checkFront (.cu:420-869, version 6): OR over the 3x3 face one cell in
     * front of the moved monomer, i.e. at r0 + 2*D along the move axis and
     * -1..+1 along the two other axes. */
    bool front(const std::vector<uint8_t> &lat, int64_t x0, int64_t y0, int64_t z0, int dir) const
    {
        const int axis = dir >> 1;
        const int s2 = (dir & 1) ? 2 : -2;
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b) {
                int64_t x = x0, y = y0, zz = z0;
                if (axis == 0) { x += s2; y += a; zz += b; }
                else if (axis == 1) { y += s2; x += a; zz += b; }
                else { zz += s2; x += a; y += b; }
                if (lat[z(x, y, zz)]) return true;
            }
        return false;
    }

    /* checkFront of the reference's perform count (.cu:1213): the nine
     * face sites' Z-order indices used as byte indices into the bit-packed
     * temporary lattice of L^3/8 bytes -- byte b holds the target bits of
     * sites 8b .. 8b+7 -- with fetches past its end reading zero (a linear
     * texture of that size, .cu:2226-2240). */
    bool front_bytes(int64_t x0, int64_t y0, int64_t z0, int dir) const
    {
        const int axis = dir >> 1;
        const int s2 = (dir & 1) ? 2 : -2;
        const uint64_t nbytes = (uint64_t)Lx * Ly * Lz / 8;
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b) {
                int64_t x = x0, y = y0, zz = z0;
                if (axis == 0) { x += s2; y += a; zz += b; }
                else if (axis == 1) { y += s2; x += a; zz += b; }
                else { zz += s2; x += a; y += b; }
                const uint64_t byte = z(x, y, zz);
                if (byte >= nbytes) continue;
                for (int k = 0; k < 8; ++k)
                    if (tmp[8 * byte + k]) return true;
            }
        return false;
    }

    uint32_t draw(uint32_t seed, uint64_t iteration, uint32_t local) const
    {
        if (rng == RNG_INTHASH) return hash_rng(seed, local);
        if (rng == RNG_PHILOX) return philox4x32_10(seed, local, iteration);
        return saru_u32(seed, (uint32_t)iteration, local);
    }

    /* kernelCountFilteredCheck (.cu:1033-1097) for one monomer and
     * direction: the move leaves the box ([0], which the reference never
     * counts); inside the box, a bond becomes invalid ([1]) and,
     * independently, the leading face is occupied ([2]). */
    void filter_tests(uint32_t id, int dir, bool &out, bool &bad, bool &occ) const
    {
        const int64_t x1 = px[id] + DX[dir], y1 = py[id] + DY[dir], z1 = pz[id] + DZ[dir];
        out = (!periodic[0] && !inside(px[id], x1, Lx)) || (!periodic[1] && !inside(py[id], y1, Ly)) ||
              (!periodic[2] && !inside(pz[id], z1, Lz));
        if (out) return;
        for (uint32_t j = 0; j < nnbr[id] && !bad; ++j) {
            const uint32_t nb = nbr[(size_t)id * 8 + j];
            bad = forbidden[bond_index(px[nb] - x1, py[nb] - y1, pz[nb] - z1)] != 0;
        }
        occ = front(lattice, px[id], py[id], pz[id], dir);
    }

    /* one colour substep: kernelSimulationScBFMCheckSpecies (.cu:930-1028)
     * followed by kernelSimulationScBFMPerformSpeciesAndApply (.cu:1148-1190)
     * with a clean temporary lattice (.cu:3050-3062, :3199-3209). */
    void substep(uint32_t sp, uint32_t seed, uint64_t iteration)
    {
        const std::vector<uint32_t> &ids = slab[sp];
        const long long m = (long long)ids.size();
        flags.assign(m, 0);
        target.assign(m, 0);
        uint64_t nc = 0, na = 0;
        /* filter counts, kernelCountFilteredCheck (.cu:1033-1097) and
         * kernelCountFilteredPerform (.cu:1192-1216): [0] walls (counted
         * here, never by the reference), [1] invalid bond, [2] occupied
         * front, [3] occupied front with valid bonds, [4] parallel refusal */
        uint64_t f0 = 0, f1 = 0, f2 = 0, f3 = 0, f4 = 0;
#pragma omp parallel for num_threads(nThreads) reduction(+ : nc, f0, f1, f2, f3) schedule(static)
        for (long long i = 0; i < m; ++i) {
            const uint32_t id = ids[i];
            const uint32_t rn = draw(seed, iteration, (uint32_t)i);
            const int dir = (int)(rn % 6u);
            if (filterStats) {
                /* the reference's count kernel draws IntHash directions whatever the RNG */
                const int dc = filterStats == 1 ? (int)(hash_rng(seed, (uint32_t)i) % 6u) : dir;
                bool out = false, bad = false, occ = false;
                filter_tests(id, dc, out, bad, occ);
                f0 += out;
                f1 += bad;
                f2 += occ;
                f3 += occ && !bad;
            }
            const int64_t x1 = px[id] + DX[dir], y1 = py[id] + DY[dir], z1 = pz[id] + DZ[dir];
            if ((!periodic[0] && !inside(px[id], x1, Lx)) || (!periodic[1] && !inside(py[id], y1, Ly)) ||
                (!periodic[2] && !inside(pz[id], z1, Lz)))
                continue;
            bool bad = false;
            for (uint32_t j = 0; j < nnbr[id] && !bad; ++j) {
                const uint32_t nb = nbr[(size_t)id * 8 + j];
                if (forbidden[bond_index(px[nb] - x1, py[nb] - y1, pz[nb] - z1)]) bad = true;
            }
            if (bad) continue;
            if (front(lattice, px[id], py[id], pz[id], dir)) continue;
            flags[i] = (uint8_t)(dir | 8);
            target[i] = z(x1, y1, z1);
            __atomic_store_n(&tmp[target[i]], (uint8_t)1, __ATOMIC_RELAXED);
            ++nc;
        }
#pragma omp parallel for num_threads(nThreads) reduction(+ : na, f4) schedule(static)
        for (long long i = 0; i < m; ++i) {
            if (!(flags[i] & 8)) continue;
            const uint32_t id = ids[i];
            const int dir = flags[i] & 7;
            const bool refused = front(tmp, px[id], py[id], pz[id], dir);
            if (filterStats == 1) {
                /* kernelCountFilteredPerform runs after the perform-and-apply
                 * kernel has moved the monomer (.cu:3163-3197) and reads the
                 * bit-packed temporary lattice (UpdaterGPUScBFM_AB_Type.h:30)
                 * with checkFront's byte fetch (.cu:420-428, :1213) */
                if (refused) f4 += front_bytes(px[id], py[id], pz[id], dir);
                else f4 += front_bytes(px[id] + DX[dir], py[id] + DY[dir], pz[id] + DZ[dir], dir);
            } else {
                f4 += refused;
            }
            if (refused) continue;
            lattice[z(px[id], py[id], pz[id])] = 0;
            px[id] += DX[dir];
            py[id] += DY[dir];
            pz[id] += DZ[dir];
            lattice[z(px[id], py[id], pz[id])] = 1;
            ++na;
        }
        /* clear the temporary lattice: only candidate targets were set */
#pragma omp parallel for num_threads(nThreads) schedule(static)
        for (long long i = 0; i < m; ++i)
            if (flags[i] & 8) __atomic_store_n(&tmp[target[i]], (uint8_t)0, __ATOMIC_RELAXED);
        nAttempt += (uint64_t)m;
        nCandidate += nc;
        nAccept += na;
        if (filterStats) { /* .cu:3316-3330 */
            const double x[5] = {(double)f0, (double)f1, (double)f2, (double)f3, (double)f4};
            for (int f = 0; f < 5; ++f) {
                const size_t at = (size_t)sp * 5 + f;
                fsum[at] += x[f];
                fsum2[at] += x[f] * x[f];
                fmin[at] = std::min(fmin[at], x[f]);
                fmax[at] = std::max(fmax[at], x[f]);
                fcnt[at] += 1.0;
            }
        }
    }

    /* runSimulationOnGPU (.cu:2902-3400) */
    void run(uint32_t nMCS, R250State &r250)
    {
        if (filterStats) { /* fresh per call (.cu:2926-2936) */
            const size_t z = (size_t)nSpecies * 5;
            fsum.assign(z, 0.0);
            fsum2.assign(z, 0.0);
            fmin.assign(z, (double)n);
            fmax.assign(z, 0.0);
            fcnt.assign(z, 0.0);
        }
        for (uint32_t iStep = 0; iStep < nMCS; ++iStep, ++age) {
            if (age % sortEvery == 0) spatialSort();
            for (uint32_t iSub = 0; iSub < nSpecies; ++iSub) {
                /* .cu:3049: mAge has already been advanced by iStep */
                const uint64_t currentAge = (uint64_t)age + (uint64_t)iStep * nSpecies + iSub;
                const uint32_t sp = (uint32_t)((uint64_t)r250_next(r250) % nSpecies);
                const uint32_t seed = r250_next(r250);
                substep(sp, seed, currentAge);
            }
        }
    }
};

} // namespace orc

using namespace orc;

/* ================================================================ C ABI === */
extern "C" {

uint32_t orc_saru(uint32_t seed, uint32_t iteration, uint32_t subseq) { return saru_u32(seed, iteration, subseq); }

/* setPeriodicity of the emulated updater (before the first run) */
void orc_sweep_set_periodicity(void *h, int px, int py, int pz)
{
    auto *s = static_cast<Sweep *>(h);
    s->periodic[0] = px != 0;
    s->periodic[1] = py != 0;
    s->periodic[2] = pz != 0;
}
uint32_t orc_hash_rng(uint32_t seed, uint32_t subseq) { return hash_rng(seed, subseq); }
uint32_t orc_philox(uint64_t seed, uint64_t subseq, uint64_t offset) { return philox4x32_10(seed, subseq, offset); }
uint32_t orc_zindex(int64_t x, int64_t y, int64_t z, uint32_t mx, uint32_t my, uint32_t mz) { return zindex(x, y, z, mx, my, mz); }

void orc_r250_seed_u64(uint32_t *state251, uint64_t seed)
{
    R250State s;
    r250_seed_u64(s, seed);
    std::memcpy(state251, s.buf, sizeof(s.buf));
    state251[250] = s.idx;
}
void orc_r250_seed_words(uint32_t *state251, const uint32_t *words250)
{
    R250State s;
    r250_seed_words(s, words250);
    std::memcpy(state251, s.buf, sizeof(s.buf));
    state251[250] = s.idx;
}
void orc_r250_draw(uint32_t *state251, uint32_t *out, size_t n)
{
    R250State s;
    std::memcpy(s.buf, state251, sizeof(s.buf));
    s.idx = state251[250];
    for (size_t i = 0; i < n; ++i) out[i] = r250_next(s);
    std::memcpy(state251, s.buf, sizeof(s.buf));
    state251[250] = s.idx;
}

/* colors_out[n]; returns number of colours or -1 on error */
int orc_graph_coloring(uint32_t n, const uint32_t *nnbr, const uint32_t *nbr8, int uniform, uint32_t *colors_out)
{
    try {
        auto c = graph_coloring(n, nnbr, nbr8, uniform != 0);
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            colors_out[i] = c[i];
            k = std::max(k, c[i] + 1);
        }
        return (int)k;
    } catch (...) {
        return -1;
    }
}

/* Stateful emulator mirroring the updater life cycle: create = setters +
 * initialize (.cu:2393-2537), run = runSimulationOnGPU, get = copy-back. */
void *orc_sweep_create(uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, const int32_t *pos3, const uint32_t *nnbr,
                       const uint32_t *nbr8, const uint8_t *forbidden512, int rng, int64_t age, int64_t sortEvery,
                       int nThreads)
{
    try {
        /* the reference takes power-of-two boxes; the batched ensembles also
         * take edges that are multiples of 8 */
        uint32_t P[3] = {1, 1, 1};
        bool pow2 = true;
        for (int a = 0; a < 3; ++a) {
            const uint32_t L = a == 0 ? Lx : (a == 1 ? Ly : Lz);
            if (L < 8 || L > 1024 || (L % 8)) return nullptr;
            while (P[a] < L) P[a] <<= 1;
            pow2 = pow2 && P[a] == L;
        }
        auto *s = new Sweep();
        s->Lx = Lx; s->Ly = Ly; s->Lz = Lz;
        s->mx = P[0] - 1; s->my = P[1] - 1; s->mz = P[2] - 1;
        s->pow2 = pow2;
        s->n = n;
        s->nnbr.assign(nnbr, nnbr + n);
        s->nbr.assign(nbr8, nbr8 + (size_t)n * 8);
        std::memcpy(s->forbidden, forbidden512, 512);
        s->rng = rng;
        s->age = age;
        s->sortEvery = sortEvery;
        s->nThreads = nThreads > 0 ? nThreads : 1;
        s->px.resize(n); s->py.resize(n); s->pz.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            s->px[i] = pos3[3 * i];
            s->py[i] = pos3[3 * i + 1];
            s->pz[i] = pos3[3 * i + 2];
        }
        s->color = graph_coloring(n, nnbr, nbr8, true);
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) k = std::max(k, s->color[i] + 1);
        s->nSpecies = k;
        s->slab.assign(k, {});
        for (uint32_t i = 0; i < n; ++i) s->slab[s->color[i]].push_back(i); /* .cu:1648-1650 */
        const uint32_t Lm = std::max(P[0], std::max(P[1], P[2]));
        const size_t sites = (size_t)Lm * Lm * Lm;
        s->lattice.assign(sites, 0);
        s->tmp.assign(sites, 0);
        for (uint32_t i = 0; i < n; ++i) s->lattice[s->z(s->px[i], s->py[i], s->pz[i])] = 1; /* .cu:2164-2171 */
        if (s->age != 0) s->spatialSort(); /* .cu:2511-2512 */
        return s;
    } catch (...) {
        return nullptr;
    }
}

void orc_sweep_destroy(void *h) { delete (Sweep *)h; }

void orc_sweep_run(void *h, uint32_t nMCS, uint32_t *state251)
{
    auto *s = (Sweep *)h;
    R250State r;
    std::memcpy(r.buf, state251, sizeof(r.buf));
    r.idx = state251[250];
    s->run(nMCS, r);
    std::memcpy(state251, r.buf, sizeof(r.buf));
    state251[250] = r.idx;
}

void orc_sweep_get(void *h, int32_t *pos3)
{
    auto *s = (Sweep *)h;
    for (uint32_t i = 0; i < s->n; ++i) {
        pos3[3 * i] = (int32_t)s->px[i];
        pos3[3 * i + 1] = (int32_t)s->py[i];
        pos3[3 * i + 2] = (int32_t)s->pz[i];
    }
}

int64_t orc_sweep_age(void *h) { return ((Sweep *)h)->age; }
uint32_t orc_sweep_nspecies(void *h) { return ((Sweep *)h)->nSpecies; }
void orc_sweep_colors(void *h, uint32_t *out)
{
    auto *s = (Sweep *)h;
    std::memcpy(out, s->color.data(), sizeof(uint32_t) * s->n);
}
/* slot order of species sp (original ids), after the latest spatial sort */
uint32_t orc_sweep_slab(void *h, uint32_t sp, uint32_t *out)
{
    auto *s = (Sweep *)h;
    if (out) std::memcpy(out, s->slab[sp].data(), sizeof(uint32_t) * s->slab[sp].size());
    return (uint32_t)s->slab[sp].size();
}
/* the reference's "Stats" filter analysis: on/off, and per species and
 * filter the min, mean, stddev (.cu:3363-3366), max and number of substeps
 * of the latest run */
void orc_sweep_set_filter_stats(void *h, int mode) { ((Sweep *)h)->filterStats = mode; }
void orc_sweep_filter_stats(void *h, double *out)
{
    auto *s = (Sweep *)h;
    for (size_t i = 0; i < (size_t)s->nSpecies * 5; ++i) {
        double *o = out + 5 * i;
        const double n = i < s->fcnt.size() ? s->fcnt[i] : 0.0;
        o[4] = n;
        if (n == 0.0) {
            o[0] = o[1] = o[2] = o[3] = 0.0;
            continue;
        }
        const double mean = s->fsum[i] / n, sum2 = s->fsum2[i] / n;
        o[0] = s->fmin[i];
        o[1] = mean;
        o[2] = std::sqrt(n / (n - 1.0) * (sum2 - mean * mean)); /* NaN when n == 1 */
        o[3] = s->fmax[i];
    }
}
void orc_sweep_stats(void *h, uint64_t *out3)
{
    auto *s = (Sweep *)h;
    out3[0] = s->nAttempt;
    out3[1] = s->nCandidate;
    out3[2] = s->nAccept;
}

/* -------------------------------------------- serial (random-sequential) BFM
 * The statistical reference: LeMonADE's serial updater (UpdaterSimpleSimulator
 * with MoveLocalSc) is not in the reference tree, so this is a plain
 * Metropolis BFM written from the model definition: pick a random monomer and
 * one of the 6 unit moves, accept if all bonds stay in the bond set and the
 * 2x2x2 cube does not overlap another one.  One MCS = n attempts. */
static inline uint64_t xs_next(uint64_t &s)
{
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

uint64_t orc_serial_run(uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, int32_t *pos3, const uint32_t *nnbr,
                        const uint32_t *nbr8, const uint8_t *forbidden512, uint64_t nMCS, uint64_t seed)
{
    for (uint32_t L : {Lx, Ly, Lz})
        if (L < 8 || L > 1024 || (L & (L - 1))) return 0; /* power-of-two boxes only */
    const uint32_t mx = Lx - 1, my = Ly - 1, mz = Lz - 1;
    const uint32_t Lm = std::max(Lx, std::max(Ly, Lz));
    std::vector<uint8_t> lat((size_t)Lm * Lm * Lm, 0);
    for (uint32_t i = 0; i < n; ++i) lat[zindex(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2], mx, my, mz)] = 1;
    uint64_t st = seed ? seed : 0x9E3779B97F4A7C15ull;
    uint64_t accepted = 0;
    const uint64_t total = nMCS * (uint64_t)n;
    for (uint64_t t = 0; t < total; ++t) {
        const uint64_t r = xs_next(st);
        const uint32_t id = (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
        const int dir = (int)((r & 0xFFFFFFFFull) % 6ull);
        int32_t *p = pos3 + 3 * (size_t)id;
        const int64_t x1 = p[0] + DX[dir], y1 = p[1] + DY[dir], z1 = p[2] + DZ[dir];
        bool bad = false;
        for (uint32_t j = 0; j < nnbr[id] && !bad; ++j) {
            const int32_t *q = pos3 + 3 * (size_t)nbr8[(size_t)id * 8 + j];
            if (forbidden512[bond_index(q[0] - x1, q[1] - y1, q[2] - z1)]) bad = true;
        }
        if (bad) continue;
        const int axis = dir >> 1;
        const int s2 = (dir & 1) ? 2 : -2;
        for (int a = -1; a <= 1 && !bad; ++a)
            for (int b = -1; b <= 1 && !bad; ++b) {
                int64_t x = p[0], y = p[1], zz = p[2];
                if (axis == 0) { x += s2; y += a; zz += b; }
                else if (axis == 1) { y += s2; x += a; zz += b; }
                else { zz += s2; x += a; y += b; }
                if (lat[zindex(x, y, zz, mx, my, mz)]) bad = true;
            }
        if (bad) continue;
        lat[zindex(p[0], p[1], p[2], mx, my, mz)] = 0;
        p[0] = (int32_t)x1; p[1] = (int32_t)y1; p[2] = (int32_t)z1;
        lat[zindex(x1, y1, z1, mx, my, mz)] = 1;
        ++accepted;
    }
    return accepted;
}

} /* extern "C" */
