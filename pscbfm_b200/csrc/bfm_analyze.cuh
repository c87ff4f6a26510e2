/*
 * bfm_analyze.cuh -- chain observables on the device between sweeps: the
 * quantities of the reference's AnalyzerMsd (src/AnalyzerMsd.tpp) for
 * systems of linear chains.
 *
 *   chain discovery (host, once): AnalyzerMsd::getLinearPolymerSystemInfo
 *     (AnalyzerMsd.tpp:193-280): chains in order of their lowest monomer id,
 *     found by a stack walk from it; the end monomers in the order the walk
 *     meets them; the middle monomer floor(n/2) bonds from the first end.
 *   per evaluation (device): end-to-end vector, radius of gyration and
 *     centre of mass of every chain from exact 64-bit integer sums of the
 *     unfolded positions; the box centre of mass as the mean of the chain
 *     centres (AnalyzerMsd.tpp:345-348); the five mean-square displacements
 *     against a recorded time origin (AnalyzerMsd.tpp:392-421): g1 first
 *     monomer, g2 middle monomer, g3 last monomer, g4 chain centre of mass
 *     -- each minus the drift of the box centre of mass when there is more
 *     than one chain -- and g5 the middle monomer relative to its chain's
 *     centre of mass.
 *
 * The block-level sums run in a fixed order, so results are reproducible
 * run to run; per-chain R_e^2 and the numerator of R_g^2 are exact integers.
 */
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace bfm {

/* linear chains of a bond graph (n x 8 neighbour ids, insertion order) by
 * the reference analyzer's rule; throws std::invalid_argument for a graph
 * that is not a set of linear chains, std::runtime_error where the
 * reference's middle-monomer walk fails */
struct LinearChains {
    std::vector<uint32_t> first, middle, last; /* monomer ids per chain */
    std::vector<uint32_t> off, members;        /* CSR: members of chain c are members[off[c] .. off[c+1]) */
};

inline LinearChains linear_chains(uint32_t n, const uint8_t *deg, const uint32_t *nbr8)
{
    LinearChains lc;
    std::vector<char> visited(n, 0);
    std::vector<uint32_t> todo;
    lc.off.push_back(0);
    for (uint32_t i0 = 0; i0 < n; ++i0) {
        if (visited[i0]) continue;
        std::vector<uint32_t> ends;
        todo.assign(1, i0);
        visited[i0] = 1;
        uint32_t count = 1;
        lc.members.push_back(i0);
        while (!todo.empty()) {
            const uint32_t m = todo.back();
            todo.pop_back();
            const uint32_t nn = deg[m];
            if (nn > 2)
                throw std::invalid_argument("Some monomers have more than two bonds: the chain analysis works with linear chains only");
            if (nn <= 1) ends.push_back(m);
            for (uint32_t b = 0; b < nn; ++b) {
                const uint32_t q = nbr8[(size_t)m * 8 + b];
                if (!visited[q]) {
                    ++count;
                    visited[q] = 1;
                    todo.push_back(q);
                    lc.members.push_back(q);
                }
            }
        }
        if (count == 1 && ends.size() == 1) ends.push_back(ends[0]);
        if (ends.size() != 2)
            throw std::invalid_argument("Found not exactly 2 end monomers in a chain (rings or loops are not linear chains)");
        uint32_t mid = ends[0], prev = mid;
        for (uint32_t s = 0; s < count / 2; ++s) {
            const uint32_t next = nbr8[(size_t)mid * 8 + 0] != prev ? nbr8[(size_t)mid * 8 + 0] : nbr8[(size_t)mid * 8 + 1];
            prev = mid;
            mid = next;
            if (deg[mid] < 2)
                throw std::runtime_error("Unexpected end monomer met while walking to the middle monomer of a chain");
        }
        lc.first.push_back(ends[0]);
        lc.middle.push_back(mid);
        lc.last.push_back(ends[1]);
        lc.off.push_back((uint32_t)lc.members.size());
    }
    return lc;
}

/* per-chain integer sums of the unfolded positions: sx, sy, sz, sum of r^2 */
struct ChainSums {
    long long sx, sy, sz, sq;
};

/* one warp per chain */
__global__ void k_chain_sums(const int32_t *__restrict__ xyz, const uint32_t *__restrict__ off,
                             const uint32_t *__restrict__ members, uint32_t nchains, ChainSums *__restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchains; c += (gridDim.x * blockDim.x) >> 5) {
        long long sx = 0, sy = 0, sz = 0, sq = 0;
        for (uint32_t j = off[c] + lane; j < off[c + 1]; j += 32u) {
            const uint32_t m = members[j];
            const long long x = xyz[3 * (size_t)m], y = xyz[3 * (size_t)m + 1], z = xyz[3 * (size_t)m + 2];
            sx += x;
            sy += y;
            sz += z;
            sq += x * x + y * y + z * z;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_down_sync(0xFFFFFFFFu, sx, o);
            sy += __shfl_down_sync(0xFFFFFFFFu, sy, o);
            sz += __shfl_down_sync(0xFFFFFFFFu, sz, o);
            sq += __shfl_down_sync(0xFFFFFFFFu, sq, o);
        }
        if (lane == 0) out[c] = ChainSums{sx, sy, sz, sq};
    }
}

/* Time origin of the mean-square displacements, per chain: first, middle
 * and last monomer, chain centre of mass, middle minus centre of mass; and
 * the box centre of mass. */
struct ChainOrigin {
    double p[5][3];
};

constexpr int kAnalyzeThreads = 1024;

__device__ __forceinline__ double block_sum(double v, double *red)
{
    /* fixed-order tree over the block: reproducible */
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = kAnalyzeThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

/* One block of kAnalyzeThreads.  out: [chains, <R_e^2>, <R_g^2>, g1..g5,
 * box COM x, y, z, end-to-end autocorrelation]; per-chain R_e^2, R_g^2 and centre of mass; with
 * setOrigin the current values become the time origin. */
__global__ void __launch_bounds__(kAnalyzeThreads)
    k_chain_observables(const int32_t *__restrict__ xyz, const ChainSums *__restrict__ sums, const uint32_t *__restrict__ off,
                        const uint32_t *__restrict__ first, const uint32_t *__restrict__ middle,
                        const uint32_t *__restrict__ last, uint32_t nchains, ChainOrigin *origin, double *boxOrigin,
                        int haveOrigin, int setOrigin, double *re2, double *rg2, double *com, double *out)
{
    __shared__ double red[kAnalyzeThreads];
    /* pass 1: per-chain values and the box centre of mass */
    double bx = 0, by = 0, bz = 0, sre = 0, srg = 0;
    for (uint32_t c = threadIdx.x; c < nchains; c += kAnalyzeThreads) {
        const ChainSums s = sums[c];
        const long long n = (long long)(off[c + 1] - off[c]);
        const double cx = (double)s.sx / (double)n, cy = (double)s.sy / (double)n, cz = (double)s.sz / (double)n;
        const int32_t *a = xyz + 3 * (size_t)first[c], *b = xyz + 3 * (size_t)last[c];
        const long long dx = (long long)b[0] - a[0], dy = (long long)b[1] - a[1], dz = (long long)b[2] - a[2];
        const double e = (double)(dx * dx + dy * dy + dz * dz);
        /* R_g^2 = (n sum r^2 - |sum r|^2) / n^2, numerator exact */
        const double g = (double)(n * s.sq - (s.sx * s.sx + s.sy * s.sy + s.sz * s.sz)) / ((double)n * (double)n);
        re2[c] = e;
        rg2[c] = g;
        com[3 * (size_t)c] = cx;
        com[3 * (size_t)c + 1] = cy;
        com[3 * (size_t)c + 2] = cz;
        bx += cx;
        by += cy;
        bz += cz;
        sre += e;
        srg += g;
    }
    const double inv = nchains ? 1.0 / (double)nchains : 0.0;
    bx = block_sum(bx, red) * inv;
    by = block_sum(by, red) * inv;
    bz = block_sum(bz, red) * inv;
    sre = block_sum(sre, red) * inv;
    srg = block_sum(srg, red) * inv;

    /* pass 2: mean-square displacements against the origin */
    double gs[5] = {0, 0, 0, 0, 0};
    double acNum = 0, acDen = 0; /* end-to-end vector autocorrelation against the origin */
    if (haveOrigin) {
        const double dbx = nchains > 1 ? bx - boxOrigin[0] : 0.0;
        const double dby = nchains > 1 ? by - boxOrigin[1] : 0.0;
        const double dbz = nchains > 1 ? bz - boxOrigin[2] : 0.0;
        for (uint32_t c = threadIdx.x; c < nchains; c += kAnalyzeThreads) {
            const ChainOrigin o = origin[c];
            const uint32_t id[3] = {first[c], middle[c], last[c]};
            double now[5][3];
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d) now[k][d] = (double)xyz[3 * (size_t)id[k] + d];
            for (int d = 0; d < 3; ++d) {
                now[3][d] = com[3 * (size_t)c + d];
                now[4][d] = now[1][d] - now[3][d];
            }
            for (int d = 0; d < 3; ++d) {
                const double r0 = o.p[2][d] - o.p[0][d];
                acNum += (now[2][d] - now[0][d]) * r0;
                acDen += r0 * r0;
            }
            const double drift[3] = {dbx, dby, dbz};
            for (int k = 0; k < 5; ++k) {
                double q = 0;
                for (int d = 0; d < 3; ++d) {
                    const double v = now[k][d] - o.p[k][d] - (k < 4 ? drift[d] : 0.0);
                    q += v * v;
                }
                gs[k] += q;
            }
        }
    }
    for (int k = 0; k < 5; ++k) gs[k] = block_sum(gs[k], red) * inv;
    acNum = block_sum(acNum, red);
    acDen = block_sum(acDen, red);

    if (setOrigin) {
        for (uint32_t c = threadIdx.x; c < nchains; c += kAnalyzeThreads) {
            ChainOrigin o;
            const uint32_t id[3] = {first[c], middle[c], last[c]};
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d) o.p[k][d] = (double)xyz[3 * (size_t)id[k] + d];
            for (int d = 0; d < 3; ++d) {
                o.p[3][d] = com[3 * (size_t)c + d];
                o.p[4][d] = o.p[1][d] - o.p[3][d];
            }
            origin[c] = o;
        }
        if (threadIdx.x == 0) {
            boxOrigin[0] = bx;
            boxOrigin[1] = by;
            boxOrigin[2] = bz;
        }
    }
    if (threadIdx.x == 0) {
        out[0] = (double)nchains;
        out[1] = sre;
        out[2] = srg;
        for (int k = 0; k < 5; ++k) out[3 + k] = gs[k];
        out[8] = bx;
        out[9] = by;
        out[10] = bz;
        out[11] = acDen > 0.0 ? acNum / acDen : 0.0;
    }
}

} // namespace bfm
