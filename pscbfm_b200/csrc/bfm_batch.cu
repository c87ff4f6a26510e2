/*
 * bfm_batch.cu -- many independent BFM systems in one persistent launch.
 *
 * Each system keeps the single-system semantics of UpdaterGPUScBFM_AB_Type
 * (runSimulationOnGPU, UpdaterGPUScBFM_AB_Type.cu:2902-3400): its own bond
 * set, colouring and species slabs (graphColoring.tpp:160-496), its own
 * R250 stream for the colour and seed of every substep (.cu:3065-3066), the
 * RNG keys (seed, currentAge, index in the species, .cu:3049), the check and
 * perform rules (.cu:930-1028, :1148-1190) and the spatial re-sort every
 * stepsBetweenSortings MCS (.cu:3005, :1835-1943).  A system of the batch
 * therefore follows exactly the trajectory a single updater with the same
 * R250 state follows.
 *
 * Layout: the systems' monomer slots are concatenated (a system's species
 * slabs are contiguous, ascending original id inside a colour until the
 * first sort); positions are Z-order codes of the wrapped coordinates in a
 * box padded to powers of two, so edge lengths need only be multiples of 8
 * (the bond code is taken mod 8 per axis); the periodic wrap at a
 * non-power-of-two edge is a compare on the dilated coordinate.
 *
 * Kernel: one CTA per system at a time, systems taken from a queue ordered
 * by decreasing work.  The CTA runs the system's substeps back to back with
 * CTA barriers only -- no grid barrier, no spin wait.  Occupation and target
 * bit lattices of systems up to 64^3 (padded) sit in shared memory; larger
 * systems use their lattice in global memory and a per-CTA target scratch.
 * A launch advances every system to its next sorting point (or the end of
 * its budget); between launches one segmented device radix sort re-sorts
 * the systems that reached a sorting point.
 */
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfm_device.cuh"
#include "bfm_host.hpp"
#include "../../include/pscbfm_b200.h"

namespace bfm {
namespace ens {

constexpr int kThreads = 512;
constexpr uint32_t kMaxSpecies = 16;
constexpr int kInFlight = 2; /* default monomers per thread in flight in the check phase (1 and 4: autotuner candidates) */
constexpr uint32_t kSmemLatWords = 8192; /* 64^3 sites: lattice and targets of smaller systems in shared memory */
constexpr uint32_t kMaxCluster = 16;     /* CTAs of a cluster, at most */

/* one system, read-only during a launch */
struct SysDesc {
    uint32_t base;                    /* first slot */
    uint32_t n;                       /* monomers */
    uint32_t nSpecies;
    uint32_t rng;                     /* BFM_RNG_* */
    uint32_t spOff[kMaxSpecies + 1];  /* species slab offsets, relative to base */
    uint32_t latOff;                  /* first word of its occupation lattice in the pool */
    uint32_t latWords;                /* padded box: max_a(P_a)^3 / 32 */
    uint32_t m[3];                    /* dilated (P_a - 1) << a: payload mask of axis a */
    uint32_t top[3];                  /* dilated (L_a - 1) << a: last coordinate before the wrap */
    uint32_t forbidden[16];           /* bond table, interleaved bond code (zbond) */
};
constexpr int kDescWords = sizeof(SysDesc) / 4;
static_assert(sizeof(SysDesc) % 4 == 0, "SysDesc is copied word by word");

/* one system's work in one launch */
struct Work {
    int64_t age;    /* mAge at the start of the launch */
    uint32_t steps; /* MCS to run */
    uint32_t done;  /* MCS of the same run call before this launch: the
                       reference's iStep counts from the start of the call (.cu:3049) */
};

/* +1 / -1 along an axis with the periodic wrap at L (payload mask m,
 * dilated L-1 in top); for power-of-two L this is the plain masked step */
__device__ __forceinline__ uint32_t winc(uint32_t a, uint32_t m, uint32_t top, uint32_t unit, bool &wrapped)
{
    const uint32_t v = a & m;
    wrapped = v == top;
    return (a & ~m) | (wrapped ? 0u : (((v | ~m) + unit) & m));
}
__device__ __forceinline__ uint32_t wdec(uint32_t a, uint32_t m, uint32_t top, uint32_t unit, bool &wrapped)
{
    const uint32_t v = a & m;
    wrapped = v == 0u;
    return (a & ~m) | (wrapped ? top : ((v - unit) & m));
}
__device__ __forceinline__ uint32_t wstep(uint32_t a, int ax, bool up, const SysDesc &s, bool &wrapped)
{
    const uint32_t m = ax == 0 ? s.m[0] : (ax == 1 ? s.m[1] : s.m[2]);
    const uint32_t t = ax == 0 ? s.top[0] : (ax == 1 ? s.top[1] : s.top[2]);
    return up ? winc(a, m, t, 1u << ax, wrapped) : wdec(a, m, t, 1u << ax, wrapped);
}
__device__ __forceinline__ uint32_t wmove(uint32_t a, int dir, const SysDesc &s, bool &wrapped)
{
    return wstep(a, dir >> 1, dir & 1, s, wrapped);
}

/* Where a system's bit lattice lives: one array (global memory, or the
 * CTA's own shared memory) ... */
struct FlatLat {
    uint32_t *p;
    __device__ __forceinline__ uint32_t *at(uint32_t w) const { return p + w; }
};
/* ... or spread over the shared memory of the cluster's CTAs: word w in the
 * CTA of rank w >> shift at index w & mask, reached through the generic
 * address of that CTA's slice (distributed shared memory) */
struct DistLat {
    uint32_t *const *rank; /* per rank: generic address of its slice */
    uint32_t shift, mask;
    __device__ __forceinline__ uint32_t *at(uint32_t w) const { return rank[w >> shift] + (w & mask); }
};

template <class LAT>
__device__ __forceinline__ bool bit(const LAT &lat, uint32_t c) { return (*lat.at(c >> 5) >> (c & 31u)) & 1u; }

/* checkFront (.cu:420-869): any of the nine sites at r0 + 2*D[dir], -1..+1
 * along the two other axes */
template <class LAT>
__device__ __forceinline__ bool face9(const LAT &lat, uint32_t r0, int dir, const SysDesc &s)
{
    bool w;
    const uint32_t c = wmove(wmove(r0, dir, s, w), dir, s, w);
    const int ax = dir >> 1, bx = ax == 0 ? 1 : 0, cx = ax == 2 ? 1 : 2;
    const uint32_t row[3] = {wstep(c, bx, false, s, w), c, wstep(c, bx, true, s, w)};
    bool any = false;
#pragma unroll
    for (int u = 0; u < 3; ++u)
        any |= bit(lat, wstep(row[u], cx, false, s, w)) | bit(lat, row[u]) | bit(lat, wstep(row[u], cx, true, s, w));
    return any;
}

/* LeMonADE's R250 (as the host R250 of this library), state in shared
 * memory: words 0..249 and the index in word 250 */
__device__ __forceinline__ uint32_t r250_next(uint32_t *st)
{
    const uint32_t i = st[250];
    const uint32_t j = i >= 147u ? i - 147u : i + 103u;
    const uint32_t v = st[i] ^ st[j];
    st[i] = v;
    st[250] = i >= 249u ? 0u : i + 1u;
    return v;
}

__device__ __forceinline__ uint32_t draw_any(uint32_t rng, uint32_t seed, uint32_t iter, uint32_t i, uint32_t iterHi)
{
    if (rng == BFM_RNG_INTHASH) return draw<RNG_INTHASH>(seed, iter, i, iterHi);
    if (rng == BFM_RNG_PHILOX) return draw<RNG_PHILOX>(seed, iter, i, iterHi);
    return draw<RNG_SARU>(seed, iter, i, iterHi);
}

struct Arrays {
    uint32_t *pos;
    int32_t *img;        /* 3 rows of T */
    const uint32_t *nbr; /* rows of T, global slot ids */
    const uint8_t *deg;
    uint8_t *flags;
    uint32_t T;
    uint32_t *latPool;
    uint32_t *tmpScratch; /* per CTA, maxLatWords each */
    uint32_t maxLatWords;
    uint32_t *r250;      /* 251 words per system */
    unsigned long long *counters; /* 3 per system: attempts, candidates, accepts */
};

/* every synchronisation of the phases of one system: the CTA, or the
 * whole cluster when a cluster shares the system (release/acquire at cluster
 * scope, which orders the global-memory lattice and target updates too) */
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
template <bool CL>
__device__ __forceinline__ void group_sync()
{
    if (CL)
        cluster_barrier();
    else
        __syncthreads();
}

/* wk.steps MCS of one system: this thread takes monomers first, first +
 * stride, ... of every species slab (stride = threads sharing the system);
 * the leader thread of each CTA draws the colour / seed sequence into its
 * CTA's shared copy (every CTA of a cluster draws the same sequence) */
template <bool CL, int IF, class LAT>
__device__ __forceinline__ void advance(const SysDesc &s, uint32_t *st, const Work wk, const LAT lat, const LAT tmp,
                                        uint32_t *clearLocal, uint32_t clearWords, uint32_t clearFirst, uint32_t clearStride,
                                        uint32_t first, uint32_t stride, const Arrays &A, uint32_t &s_sp,
                                        uint32_t &s_seed, unsigned long long &s_att, bool leader, unsigned int &myCand,
                                        unsigned int &myAcc, bool countAtt = true)
{
    const uint32_t base = s.base, nSp = s.nSpecies;
        /* colour and seed of the first substep; later ones are drawn by
         * thread 0 while the targets are cleared */
        if (leader && wk.steps) {
            s_sp = r250_next(st) % nSp; /* .cu:3065 */
            s_seed = r250_next(st);     /* .cu:3066 */
        }
        group_sync<CL>();
        for (uint32_t iStep = 0; iStep < wk.steps; ++iStep) {
            const uint64_t a = (uint64_t)(wk.age + iStep); /* mAge, advanced once per MCS (.cu:3002) */
            const uint64_t callStep = (uint64_t)wk.done + iStep;
            for (uint32_t sub = 0; sub < nSp; ++sub) {
                const uint32_t sp = s_sp, seed = s_seed;
                const uint64_t currentAge = a + callStep * nSp + sub; /* .cu:3049 */
                const uint32_t iter = (uint32_t)currentAge, iterHi = (uint32_t)(currentAge >> 32);
                const uint32_t off = base + s.spOff[sp], cnt = s.spOff[sp + 1] - s.spOff[sp];
                if (leader && countAtt) s_att += cnt;

                /* check (.cu:930-1028), IF monomers in flight per thread */
                for (uint32_t i0 = first; i0 < cnt; i0 += (uint32_t)IF * stride) {
                    uint32_t slot[IF], r0[IF], r1[IF], dg[IF];
                    int dir[IF];
                    bool live[IF], ok[IF];
#pragma unroll
                    for (int u = 0; u < IF; ++u) {
                        const uint32_t i = i0 + (uint32_t)u * stride;
                        live[u] = i < cnt;
                        slot[u] = off + (live[u] ? i : 0u);
                        r0[u] = live[u] ? A.pos[slot[u]] : 0u;
                        dg[u] = live[u] ? A.deg[slot[u]] : 0u;
                        ok[u] = live[u];
                    }
#pragma unroll
                    for (int u = 0; u < IF; ++u) {
                        dir[u] = direction(draw_any(s.rng, seed, iter, i0 + (uint32_t)u * stride, iterHi));
                        bool w;
                        r1[u] = wmove(r0[u], dir[u], s, w);
                    }
                    uint32_t dmax = 0;
#pragma unroll
                    for (int u = 0; u < IF; ++u) dmax = dg[u] > dmax ? dg[u] : dmax;
                    for (uint32_t j = 0; j < dmax; ++j) {
#pragma unroll
                        for (int u = 0; u < IF; ++u)
                            if (ok[u] && j < dg[u]) {
                                const uint32_t code = zbond(A.pos[A.nbr[(size_t)j * A.T + slot[u]]], r1[u]);
                                if ((s.forbidden[code >> 5] >> (code & 31u)) & 1u) ok[u] = false;
                            }
                    }
#pragma unroll
                    for (int u = 0; u < IF; ++u)
                        if (ok[u]) ok[u] = !face9(lat, r0[u], dir[u], s);
#pragma unroll
                    for (int u = 0; u < IF; ++u)
                        if (live[u]) {
                            if (ok[u]) {
                                atomicOr(tmp.at(r1[u] >> 5), 1u << (r1[u] & 31u));
                                ++myCand;
                            }
                            A.flags[slot[u]] = ok[u] ? (uint8_t)(dir[u] | 8) : (uint8_t)0;
                        }
                }
                group_sync<CL>();

                /* perform (.cu:1148-1190) */
                for (uint32_t i = first; i < cnt; i += stride) {
                    const uint32_t slot = off + i;
                    const uint8_t f = A.flags[slot];
                    if (!(f & 8)) continue;
                    const uint32_t r0 = A.pos[slot];
                    const int dir = f & 7;
                    if (face9(tmp, r0, dir, s)) continue;
                    bool wrapped;
                    const uint32_t r1 = wmove(r0, dir, s, wrapped);
                    const uint32_t w0 = r0 >> 5, w1 = r1 >> 5;
                    const uint32_t b0 = 1u << (r0 & 31u), b1 = 1u << (r1 & 31u);
                    if (w0 == w1) {
                        atomicXor(lat.at(w0), b0 | b1);
                    } else {
                        atomicXor(lat.at(w0), b0);
                        atomicXor(lat.at(w1), b1);
                    }
                    A.pos[slot] = r1;
                    if (wrapped) A.img[(size_t)(dir >> 1) * A.T + slot] += (dir & 1) ? 1 : -1;
                    A.flags[slot] = f | 16;
                    ++myAcc;
                }
                group_sync<CL>();

                /* clear this substep's targets: this CTA's shared-memory part
                 * of the buffer when it is in shared memory, the candidates'
                 * words otherwise */
                if (leader && !(iStep + 1 == wk.steps && sub + 1 == nSp)) {
                    s_sp = r250_next(st) % nSp;
                    s_seed = r250_next(st);
                }
                if (clearLocal) {
                    uint4 *t4 = reinterpret_cast<uint4 *>(clearLocal);
                    for (uint32_t w = clearFirst; w < clearWords / 4; w += clearStride) t4[w] = make_uint4(0u, 0u, 0u, 0u);
                } else {
                    for (uint32_t i = first; i < cnt; i += stride) {
                        const uint32_t slot = off + i;
                        const uint8_t f = A.flags[slot];
                        if (!(f & 8)) continue;
                        bool w;
                        const uint32_t r1 = (f & 16) ? A.pos[slot] : wmove(A.pos[slot], f & 7, s, w);
                        *tmp.at(r1 >> 5) = 0u;
                    }
                }
                group_sync<CL>();
            }
        }

}

template <int IF>
__global__ void __launch_bounds__(kThreads, 2)
    k_batch(const SysDesc *__restrict__ desc, const Work *__restrict__ work, const uint32_t *__restrict__ order,
            uint32_t nOrder, unsigned int *next, Arrays A)
{
    extern __shared__ uint32_t dyn[]; /* kSmemLatWords occupation + kSmemLatWords targets */
    __shared__ SysDesc s;
    __shared__ uint32_t st[251];
    __shared__ uint32_t s_item, s_sp, s_seed;
    __shared__ unsigned long long s_cand, s_acc, s_att;
    const uint32_t tid = threadIdx.x;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(next, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= nOrder) return;
        const uint32_t sid = order[item];
        for (uint32_t w = tid; w < (uint32_t)kDescWords; w += blockDim.x)
            reinterpret_cast<uint32_t *>(&s)[w] = reinterpret_cast<const uint32_t *>(desc + sid)[w];
        for (uint32_t w = tid; w < 251u; w += blockDim.x) st[w] = A.r250[(size_t)sid * 251 + w];
        if (tid == 0) {
            s_cand = 0;
            s_acc = 0;
            s_att = 0;
        }
        __syncthreads();
        const uint32_t lw = s.latWords;
        const bool inSmem = lw <= kSmemLatWords;
        uint32_t *lat = inSmem ? dyn : A.latPool + s.latOff;
        uint32_t *tmp = inSmem ? dyn + kSmemLatWords : A.tmpScratch + (size_t)blockIdx.x * A.maxLatWords;
        for (uint32_t w = tid; w < lw; w += blockDim.x) {
            if (inSmem) lat[w] = A.latPool[s.latOff + w];
            tmp[w] = 0u;
        }
        __syncthreads();

        const Work wk = work[sid];
        unsigned int myCand = 0, myAcc = 0;
        advance<false, IF>(s, st, wk, FlatLat{lat}, FlatLat{tmp}, inSmem ? tmp : nullptr, lw, tid, blockDim.x, tid, blockDim.x, A,
                           s_sp, s_seed, s_att, tid == 0, myCand, myAcc);

        /* write back */
        atomicAdd(&s_cand, (unsigned long long)myCand);
        atomicAdd(&s_acc, (unsigned long long)myAcc);
        if (inSmem)
            for (uint32_t w = tid; w < lw; w += blockDim.x) A.latPool[s.latOff + w] = lat[w];
        for (uint32_t w = tid; w < 251u; w += blockDim.x) A.r250[(size_t)sid * 251 + w] = st[w];
        __syncthreads();
        if (tid == 0) {
            A.counters[3 * (size_t)sid + 0] += s_att;
            A.counters[3 * (size_t)sid + 1] += s_cand;
            A.counters[3 * (size_t)sid + 2] += s_acc;
        }
        __syncthreads();
    }
}

/* Systems whose lattice is in global memory, shared by a cluster of CTAs
 * (2, 4 or 8, chosen at launch): the cluster takes one system at a time from
 * its own queue and splits every species slab over its CTAs; phases are
 * separated by hardware cluster barriers (no spin wait).  The system's
 * target lattice is the cluster's slice of the scratch. */

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_size()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_index()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}

/* generic address of the same shared-memory location in CTA `r` of the cluster */
__device__ __forceinline__ uint32_t *cluster_map(uint32_t *p, uint32_t r)
{
    uint64_t q;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(q) : "l"(p), "r"(r));
    return reinterpret_cast<uint32_t *>(q);
}

template <int IF>
__global__ void __launch_bounds__(kThreads, 2)
    k_batch_cl(const SysDesc *__restrict__ desc, const Work *__restrict__ work, const uint32_t *__restrict__ order,
               uint32_t nOrder, unsigned int *next, uint32_t *clusterItem, Arrays A)
{
    extern __shared__ uint32_t dyn[]; /* this CTA's slices: kSmemLatWords occupation + kSmemLatWords targets */
    __shared__ SysDesc s;
    __shared__ uint32_t st[251];
    __shared__ uint32_t s_sp, s_seed;
    __shared__ unsigned long long s_cand, s_acc, s_att;
    __shared__ uint32_t *s_latRank[kMaxCluster], *s_tmpRank[kMaxCluster];
    const uint32_t tid = threadIdx.x, rank = cluster_rank(), cid = cluster_index(), cs = cluster_size();
    const uint32_t first = rank * blockDim.x + tid, stride = cs * blockDim.x;
    if (tid < cs) {
        s_latRank[tid] = cluster_map(dyn, tid);
        s_tmpRank[tid] = cluster_map(dyn + kSmemLatWords, tid);
    }

    for (;;) {
        if (rank == 0 && tid == 0) clusterItem[cid] = atomicAdd(next, 1u);
        cluster_barrier();
        const uint32_t item = *reinterpret_cast<volatile const uint32_t *>(clusterItem + cid);
        cluster_barrier(); /* every CTA has read the item before the next one is taken */
        if (item >= nOrder) return;
        const uint32_t sid = order[item];
        for (uint32_t w = tid; w < (uint32_t)kDescWords; w += blockDim.x)
            reinterpret_cast<uint32_t *>(&s)[w] = reinterpret_cast<const uint32_t *>(desc + sid)[w];
        for (uint32_t w = tid; w < 251u; w += blockDim.x) st[w] = A.r250[(size_t)sid * 251 + w];
        if (tid == 0) {
            s_cand = 0;
            s_acc = 0;
            s_att = 0;
        }
        __syncthreads();
        const uint32_t lw = s.latWords;
        const Work wk = work[sid];
        unsigned int myCand = 0, myAcc = 0;
        /* the lattices in the cluster's distributed shared memory when each
         * CTA's share fits its slices, else in global memory */
        const uint32_t slice = lw / cs;
        if (slice * cs == lw && slice <= kSmemLatWords && (slice & (slice - 1)) == 0 && slice >= 4) {
            const uint32_t *g = A.latPool + s.latOff + (size_t)rank * slice;
            for (uint32_t w = tid; w < slice; w += blockDim.x) {
                dyn[w] = g[w];
                dyn[kSmemLatWords + w] = 0u;
            }
            cluster_barrier();
            const uint32_t sh = 31u - __clz(slice);
            advance<true, IF>(s, st, wk, DistLat{s_latRank, sh, slice - 1u}, DistLat{s_tmpRank, sh, slice - 1u},
                              dyn + kSmemLatWords, slice, tid, blockDim.x, first, stride, A, s_sp, s_seed, s_att, tid == 0,
                              myCand, myAcc, rank == 0);
            uint32_t *gw = A.latPool + s.latOff + (size_t)rank * slice;
            for (uint32_t w = tid; w < slice; w += blockDim.x) gw[w] = dyn[w];
        } else {
            uint32_t *lat = A.latPool + s.latOff;
            uint32_t *tmp = A.tmpScratch + (size_t)cid * A.maxLatWords;
            for (uint32_t w = first; w < lw; w += stride) tmp[w] = 0u;
            cluster_barrier();
            advance<true, IF>(s, st, wk, FlatLat{lat}, FlatLat{tmp}, nullptr, 0u, 0u, 1u, first, stride, A, s_sp, s_seed, s_att,
                              tid == 0, myCand, myAcc, rank == 0);
        }
        atomicAdd(&s_cand, (unsigned long long)myCand);
        atomicAdd(&s_acc, (unsigned long long)myAcc);
        if (rank == 0)
            for (uint32_t w = tid; w < 251u; w += blockDim.x) A.r250[(size_t)sid * 251 + w] = st[w];
        __syncthreads();
        if (tid == 0) {
            if (rank == 0) atomicAdd(A.counters + 3 * (size_t)sid + 0, s_att);
            atomicAdd(A.counters + 3 * (size_t)sid + 1, s_cand);
            atomicAdd(A.counters + 3 * (size_t)sid + 2, s_acc);
        }
        cluster_barrier();
    }
}

/* sort keys: (segment, Z-order code) for systems due for a re-sort,
 * (segment, current index) for the others, which keeps their order */
__global__ void k_sort_keys(const uint32_t *__restrict__ pos, const uint32_t *__restrict__ slotSeg,
                            const uint32_t *__restrict__ segStart, const uint8_t *__restrict__ segSort, uint32_t T,
                            unsigned long long *__restrict__ keys, uint32_t *__restrict__ iota)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        const uint32_t g = slotSeg[i];
        const uint32_t k = segSort[g] ? pos[i] : i - segStart[g];
        keys[i] = ((unsigned long long)g << 32) | k;
        iota[i] = i;
    }
}

__global__ void k_inv(const uint32_t *__restrict__ perm, uint32_t *__restrict__ inv, uint32_t T)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) inv[perm[i]] = i;
}

__global__ void k_perm(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ inv, uint32_t T, uint32_t rows,
                       const uint32_t *__restrict__ pos, const int32_t *__restrict__ img, const uint32_t *__restrict__ nbr,
                       const uint8_t *__restrict__ deg, const uint32_t *__restrict__ s2o, uint32_t *__restrict__ pos2,
                       int32_t *__restrict__ img2, uint32_t *__restrict__ nbr2, uint8_t *__restrict__ deg2,
                       uint32_t *__restrict__ s2o2)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        const uint32_t p = perm[i];
        pos2[i] = pos[p];
        for (int a = 0; a < 3; ++a) img2[(size_t)a * T + i] = img[(size_t)a * T + p];
        const uint8_t d = deg[p];
        deg2[i] = d;
        for (uint32_t j = 0; j < rows; ++j) nbr2[(size_t)j * T + i] = j < d ? inv[nbr[(size_t)j * T + p]] : 0u;
        s2o2[i] = s2o[p];
    }
}

/* unfolded positions of one system in its original monomer order */
__global__ void k_unfold(const uint32_t *__restrict__ pos, const int32_t *__restrict__ img, const uint32_t *__restrict__ s2o,
                         uint32_t T, uint32_t base, uint32_t n, int32_t Lx, int32_t Ly, int32_t Lz, int32_t *__restrict__ out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = base + i, o = s2o[slot], c = pos[slot];
        out[3 * (size_t)o + 0] = (int32_t)undilate3(c) + img[slot] * Lx;
        out[3 * (size_t)o + 1] = (int32_t)undilate3(c >> 1) + img[(size_t)T + slot] * Ly;
        out[3 * (size_t)o + 2] = (int32_t)undilate3(c >> 2) + img[2 * (size_t)T + slot] * Lz;
    }
}

/* slot of every monomer, by global original index (system base + original id) */
__global__ void k_slot_of(const uint32_t *__restrict__ s2o, const SysDesc *__restrict__ desc, uint32_t nsys, uint32_t T,
                          uint32_t *__restrict__ slotOf)
{
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < T; slot += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nsys; /* the system whose slot range holds `slot` */
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (desc[mid].base <= slot) lo = mid;
            else hi = mid;
        }
        slotOf[desc[lo].base + s2o[slot]] = slot;
    }
}

/* unfolded positions of selected monomers: ids[k] = (system << 32) | original id */
__global__ void k_gather(const uint32_t *__restrict__ pos, const int32_t *__restrict__ img, const uint32_t *__restrict__ slotOf,
                         const SysDesc *__restrict__ desc, uint32_t T, const unsigned long long *__restrict__ ids, uint32_t m,
                         int32_t *__restrict__ out)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const unsigned long long id = ids[k];
        const SysDesc &d = desc[id >> 32];
        const uint32_t slot = slotOf[d.base + (uint32_t)id], c = pos[slot];
        out[3 * (size_t)k + 0] = (int32_t)undilate3(c) + img[slot] * (int32_t)(undilate3(d.top[0]) + 1);
        out[3 * (size_t)k + 1] = (int32_t)undilate3(c >> 1) + img[(size_t)T + slot] * (int32_t)(undilate3(d.top[1] >> 1) + 1);
        out[3 * (size_t)k + 2] = (int32_t)undilate3(c >> 2) + img[2 * (size_t)T + slot] * (int32_t)(undilate3(d.top[2] >> 2) + 1);
    }
}

/* ---------------------------------------------------------------- host */

struct Err : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaErr : Err {
    using Err::Err;
};
struct ArgErr : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

#define BCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) throw CudaErr(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
void balloc(T *&p, size_t n)
{
    p = nullptr;
    if (n) BCK(cudaMalloc((void **)&p, n * sizeof(T)));
}
template <typename T>
void bfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

uint32_t pow2_at_least(uint32_t v)
{
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

/* a system as added, before initialize */
struct Pending {
    uint32_t L[3];
    uint32_t n;
    std::vector<int32_t> xyz;
    std::vector<uint8_t> deg;
    std::vector<uint32_t> nbr; /* 8 per monomer */
    std::vector<uint8_t> allowed;
    int rng;
    int64_t age, sortEvery;
    std::vector<uint32_t> r250; /* 251 words */
};

/* the kernels of one monomers-in-flight count */
inline const void *batchKernel(int f)
{
    return f == 1 ? (const void *)k_batch<1> : f == 4 ? (const void *)k_batch<4> : (const void *)k_batch<2>;
}
inline const void *clusterKernel(int f)
{
    return f == 1 ? (const void *)k_batch_cl<1> : f == 4 ? (const void *)k_batch_cl<4> : (const void *)k_batch_cl<2>;
}

/* the autotuner's trials, in order: cluster sizes 4, 2, 8, off (2 in
 * flight); then 1 and 4 monomers in flight with the chosen size; then the
 * cluster kernel also for systems above 32^3 sites */
constexpr int kTrials = 7;
constexpr uint32_t kClusterAboveLow = 1024;

struct Batch {
    int gpu = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    bool initialized = false;
    std::vector<Pending> pend;

    /* host copies */
    std::vector<SysDesc> desc;
    std::vector<int64_t> age, sortEvery;
    std::vector<uint32_t> segOfSys; /* first segment of each system */
    uint32_t T = 0, rows = 1, nSeg = 0, maxLatWords = 0;
    size_t poolWords = 0;
    int grid = 0;

    /* device */
    SysDesc *d_desc = nullptr;
    Work *d_work = nullptr;
    uint32_t *d_order = nullptr;
    unsigned int *d_next = nullptr;
    uint32_t *d_pos = nullptr, *d_pos2 = nullptr, *d_nbr = nullptr, *d_nbr2 = nullptr, *d_s2o = nullptr, *d_s2o2 = nullptr;
    int32_t *d_img = nullptr, *d_img2 = nullptr;
    uint8_t *d_deg = nullptr, *d_deg2 = nullptr, *d_flags = nullptr;
    uint32_t *d_lat = nullptr, *d_tmp = nullptr, *d_r250 = nullptr;
    unsigned long long *d_cnt = nullptr;
    uint32_t *d_slotSeg = nullptr, *d_segStart = nullptr, *d_iota = nullptr, *d_perm = nullptr, *d_inv = nullptr;
    uint8_t *d_segSort = nullptr;
    unsigned long long *d_keys = nullptr, *d_keys2 = nullptr;
    void *d_cub = nullptr;
    size_t cubBytes = 0;
    int32_t *d_out = nullptr;
    size_t outCap = 0;
    /* selected-monomer read-back: slot of every global original index
     * (rebuilt after runs, which re-sort), requested ids and their positions */
    uint32_t *d_slotOf = nullptr;
    bool slotOfValid = false;
    unsigned long long *d_gids = nullptr;
    int32_t *d_gout = nullptr;
    size_t gCap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t stream2 = nullptr; /* the single-CTA kernel runs beside the cluster kernel */
    cudaEvent_t evFork = nullptr, evJoin = nullptr, evT0 = nullptr, evT1 = nullptr;
    uint32_t *d_clItem = nullptr;
    int clusterSize = 4;     /* CTAs per system with a global-memory lattice; 0: one CTA */
    int inFlight = kInFlight; /* monomers per thread in flight in the check phase: 1, 2 or 4 */
    uint32_t clusterAbove = kSmemLatWords; /* systems with more lattice words go to the cluster kernel */
    bool autotune = false;   /* time the launch shapes on the first launches of a run, keep the fastest */
    double tunedNs = 0;      /* ns per attempted move of the configuration chosen so far */
    bool tuned = false;
    std::vector<double> trialNsPerMove; /* per candidate of the autotuner */

    double lastMs = 0;
    uint64_t lastLaunches = 0, lastAttempts = 0;

    ~Batch() { release(); }

    void release()
    {
        if (stream) cudaStreamSynchronize(stream);
        bfree(d_desc); bfree(d_work); bfree(d_order); bfree(d_next);
        bfree(d_pos); bfree(d_pos2); bfree(d_nbr); bfree(d_nbr2); bfree(d_s2o); bfree(d_s2o2);
        bfree(d_img); bfree(d_img2); bfree(d_deg); bfree(d_deg2); bfree(d_flags);
        bfree(d_lat); bfree(d_tmp); bfree(d_r250); bfree(d_cnt);
        bfree(d_slotSeg); bfree(d_segStart); bfree(d_iota); bfree(d_perm); bfree(d_inv); bfree(d_segSort);
        bfree(d_keys); bfree(d_keys2); bfree(d_out);
        bfree(d_slotOf); bfree(d_gids); bfree(d_gout);
        gCap = 0;
        slotOfValid = false;
        if (d_cub) cudaFree(d_cub);
        d_cub = nullptr;
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evFork) cudaEventDestroy(evFork);
        if (evJoin) cudaEventDestroy(evJoin);
        if (evT0) cudaEventDestroy(evT0);
        if (evT1) cudaEventDestroy(evT1);
        ev0 = ev1 = evFork = evJoin = evT0 = evT1 = nullptr;
        bfree(d_clItem);
        if (stream2) cudaStreamDestroy(stream2);
        stream2 = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        initialized = false;
    }

    uint32_t add(const uint32_t L[3], uint32_t n, const int32_t *pos3, const uint8_t *deg, const uint32_t *nbr8,
                 const uint8_t *allowed512, int rng, int64_t a, int64_t sortEv, const uint32_t *state251, uint64_t seed)
    {
        if (initialized) throw Err("systems can only be added before bfm_batch_initialize");
        if (n == 0 || !pos3 || !deg || !nbr8 || !allowed512) throw ArgErr("a system needs monomers, bonds and a bond set");
        for (int k = 0; k < 3; ++k)
            if (L[k] < 8 || L[k] > 1024 || L[k] % 8) throw ArgErr("box edges must be multiples of 8 in 8 .. 1024");
        if (rng != BFM_RNG_INTHASH && rng != BFM_RNG_SARU && rng != BFM_RNG_PHILOX)
            throw ArgErr("random number generator must be IntHash (1), Saru (2) or Philox (3)");
        if (a < 0 || sortEv <= 0) throw ArgErr("age must be >= 0 and the sorting interval > 0");
        for (uint32_t i = 0; i < n; ++i)
            if (deg[i] > 8) throw ArgErr("at most 8 bonds per monomer (monomer " + std::to_string(i) + ")");
        Pending p;
        std::memcpy(p.L, L, sizeof(p.L));
        p.n = n;
        p.xyz.assign(pos3, pos3 + 3 * (size_t)n);
        p.deg.assign(deg, deg + n);
        p.nbr.assign(nbr8, nbr8 + 8 * (size_t)n);
        p.allowed.assign(allowed512, allowed512 + 512);
        p.rng = rng;
        p.age = a;
        p.sortEvery = sortEv;
        p.r250.resize(251);
        if (state251) {
            std::memcpy(p.r250.data(), state251, 251 * sizeof(uint32_t));
            if (p.r250[250] > 249) throw ArgErr("R250 state index must be < 250");
        } else {
            R250 r;
            r.seed_u64(seed);
            std::memcpy(p.r250.data(), r.buf, 250 * sizeof(uint32_t));
            p.r250[250] = r.idx;
        }
        pend.push_back(std::move(p));
        return (uint32_t)pend.size() - 1;
    }

    void initialize()
    {
        if (initialized) throw Err("bfm_batch_initialize was already called");
        if (pend.empty()) throw Err("no system was added");
        BCK(cudaSetDevice(gpu));
        const size_t S = pend.size();
        desc.assign(S, SysDesc{});
        age.resize(S);
        sortEvery.resize(S);
        segOfSys.resize(S + 1);
        std::vector<uint32_t> hpos, hs2o, hnbrTmp, segStart, slotSeg;
        std::vector<int32_t> himg;
        std::vector<uint8_t> hdeg, segSortInit;
        std::vector<uint32_t> hlat;
        std::vector<uint32_t> hr250(S * 251);
        rows = 1;
        for (const auto &p : pend)
            for (uint32_t i = 0; i < p.n; ++i) rows = std::max<uint32_t>(rows, p.deg[i]);
        T = 0;
        poolWords = 0;
        maxLatWords = 0;
        nSeg = 0;
        std::vector<std::vector<uint32_t>> nbrRows; /* per system: rows x n, global slot ids */
        struct Tmp {
            std::vector<uint32_t> o2s;
        };
        std::vector<Tmp> tmpv(S);
        for (size_t sI = 0; sI < S; ++sI) {
            const Pending &p = pend[sI];
            SysDesc &d = desc[sI];
            /* bond table (initializeBondTable, .cu:1516-1559): exactly 108 allowed bonds */
            unsigned nAllowed = 0;
            for (int i = 0; i < 512; ++i) nAllowed += p.allowed[i] ? 1 : 0;
            if (nAllowed != 108) throw Err("system " + std::to_string(sI) + ": expected 108 allowed bonds, got " + std::to_string(nAllowed));
            std::memset(d.forbidden, 0, sizeof(d.forbidden));
            for (uint32_t dz = 0; dz < 8; ++dz)
                for (uint32_t dy = 0; dy < 8; ++dy)
                    for (uint32_t dx = 0; dx < 8; ++dx)
                        if (!p.allowed[dx | (dy << 3) | (dz << 6)]) {
                            const uint32_t code = zcode(dx, dy, dz);
                            d.forbidden[code >> 5] |= 1u << (code & 31);
                        }
            uint32_t P[3], Pm = 0;
            for (int k = 0; k < 3; ++k) {
                P[k] = pow2_at_least(p.L[k]);
                Pm = std::max(Pm, P[k]);
                d.m[k] = dilate3(P[k] - 1) << k;
                d.top[k] = dilate3(p.L[k] - 1) << k;
            }
            d.latWords = std::max<uint32_t>(1, (uint32_t)(((uint64_t)Pm * Pm * Pm) / 32));
            d.latOff = (uint32_t)poolWords;
            poolWords += d.latWords;
            maxLatWords = std::max(maxLatWords, d.latWords);
            d.rng = (uint32_t)p.rng;
            d.n = p.n;
            d.base = T;
            for (uint32_t i = 0; i < p.n; ++i)
                for (uint32_t j = 0; j < p.deg[i]; ++j)
                    if (p.nbr[8 * (size_t)i + j] >= p.n)
                        throw ArgErr("system " + std::to_string(sI) + ": bond partner id out of range");
            /* colouring and species slabs (initializeSpeciesSorting, .cu:1561-1686) */
            const std::vector<uint32_t> color = color_graph(p.n, p.deg.data(), p.nbr.data(), true);
            uint32_t k = 0;
            for (uint32_t i = 0; i < p.n; ++i) k = std::max(k, color[i] + 1);
            if (k > kMaxSpecies) throw Err("system " + std::to_string(sI) + ": more than 16 colours");
            d.nSpecies = k;
            std::vector<uint32_t> count(k, 0);
            for (uint32_t i = 0; i < p.n; ++i) ++count[color[i]];
            d.spOff[0] = 0;
            for (uint32_t c = 0; c < k; ++c) d.spOff[c + 1] = d.spOff[c] + count[c];
            for (uint32_t c = k; c < kMaxSpecies; ++c) d.spOff[c + 1] = d.spOff[k];
            segOfSys[sI] = nSeg;
            for (uint32_t c = 0; c < k; ++c) {
                segStart.push_back(T + d.spOff[c]);
                segSortInit.push_back(0);
                for (uint32_t q = 0; q < count[c]; ++q) slotSeg.push_back(nSeg + c);
            }
            nSeg += k;
            /* slot order inside a species: ascending original id (.cu:1648-1650) */
            std::vector<uint32_t> &o2s = tmpv[sI].o2s;
            o2s.resize(p.n);
            {
                std::vector<uint32_t> nx(k);
                for (uint32_t c = 0; c < k; ++c) nx[c] = d.spOff[c];
                for (uint32_t i = 0; i < p.n; ++i) o2s[i] = nx[color[i]]++;
            }
            /* wrapped codes, image counters, lattice; excluded volume and bonds (checkSystem, .cu:2789-2900) */
            hpos.resize(T + p.n);
            hs2o.resize(T + p.n);
            hdeg.resize(T + p.n);
            himg.resize(3 * (size_t)(T + p.n)); /* per-axis rows are re-laid out below */
            hlat.resize(poolWords, 0u);
            std::vector<uint64_t> cells(((size_t)Pm * Pm * Pm + 63) / 64, 0);
            for (uint32_t i = 0; i < p.n; ++i) {
                const uint32_t slot = T + o2s[i];
                uint32_t w[3];
                for (int a = 0; a < 3; ++a) {
                    const int64_t v = p.xyz[3 * (size_t)i + a], La = p.L[a];
                    int64_t q = v / La, r = v - q * La;
                    if (r < 0) {
                        r += La;
                        --q;
                    }
                    w[a] = (uint32_t)r;
                    himg[3 * (size_t)slot + a] = (int32_t)q;
                }
                const uint32_t code = zcode(w[0], w[1], w[2]);
                hpos[slot] = code;
                hs2o[slot] = i;
                hdeg[slot] = p.deg[i];
                uint32_t *lat = hlat.data() + d.latOff;
                if ((lat[code >> 5] >> (code & 31)) & 1u)
                    throw ArgErr("system " + std::to_string(sI) + ": two monomers share the position of monomer " + std::to_string(i));
                lat[code >> 5] |= 1u << (code & 31);
                for (int c = 0; c < 8; ++c) {
                    const uint32_t cc = zcode((w[0] + (c & 1)) % p.L[0], (w[1] + ((c >> 1) & 1)) % p.L[1], (w[2] + ((c >> 2) & 1)) % p.L[2]);
                    if ((cells[cc >> 6] >> (cc & 63)) & 1u)
                        throw ArgErr("system " + std::to_string(sI) + ": excluded volume violated at monomer " + std::to_string(i));
                    cells[cc >> 6] |= 1ull << (cc & 63);
                }
            }
            for (uint32_t i = 0; i < p.n; ++i)
                for (uint32_t j = 0; j < p.deg[i]; ++j) {
                    const uint32_t o = p.nbr[8 * (size_t)i + j];
                    int64_t dv[3];
                    for (int a = 0; a < 3; ++a) dv[a] = (int64_t)p.xyz[3 * (size_t)o + a] - p.xyz[3 * (size_t)i + a];
                    bool bad = false;
                    for (int a = 0; a < 3; ++a) bad |= dv[a] < -3 || dv[a] > 3;
                    if (bad || !p.allowed[(dv[0] & 7) | ((dv[1] & 7) << 3) | ((dv[2] & 7) << 6)])
                        throw ArgErr("system " + std::to_string(sI) + ": bond " + std::to_string(i) + "-" + std::to_string(o) +
                                     " is not in the bond set");
                }
            age[sI] = p.age;
            sortEvery[sI] = p.sortEvery;
            std::memcpy(hr250.data() + sI * 251, p.r250.data(), 251 * sizeof(uint32_t));
            T += p.n;
        }
        segOfSys[S] = nSeg;
        /* neighbour rows with global slot ids */
        std::vector<uint32_t> hnbr((size_t)rows * T, 0u);
        for (size_t sI = 0; sI < S; ++sI) {
            const Pending &p = pend[sI];
            const uint32_t b = desc[sI].base;
            for (uint32_t i = 0; i < p.n; ++i) {
                const uint32_t slot = b + tmpv[sI].o2s[i];
                for (uint32_t j = 0; j < p.deg[i]; ++j) hnbr[(size_t)j * T + slot] = b + tmpv[sI].o2s[p.nbr[8 * (size_t)i + j]];
            }
        }
        std::vector<int32_t> himgRows(3 * (size_t)T);
        for (uint32_t i = 0; i < T; ++i)
            for (int a = 0; a < 3; ++a) himgRows[(size_t)a * T + i] = himg[3 * (size_t)i + a];

        BCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        BCK(cudaEventCreate(&ev0));
        BCK(cudaEventCreate(&ev1));
        BCK(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
        BCK(cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming));
        BCK(cudaEventCreateWithFlags(&evJoin, cudaEventDisableTiming));
        BCK(cudaEventCreate(&evT0));
        BCK(cudaEventCreate(&evT1));
        balloc(d_desc, S);
        balloc(d_work, S);
        balloc(d_order, S);
        balloc(d_next, 2);
        balloc(d_pos, T); balloc(d_pos2, T);
        balloc(d_img, 3 * (size_t)T); balloc(d_img2, 3 * (size_t)T);
        balloc(d_nbr, (size_t)rows * T); balloc(d_nbr2, (size_t)rows * T);
        balloc(d_deg, T); balloc(d_deg2, T);
        balloc(d_s2o, T); balloc(d_s2o2, T);
        balloc(d_flags, T);
        balloc(d_lat, poolWords);
        balloc(d_r250, S * 251);
        balloc(d_cnt, 3 * S);
        balloc(d_slotSeg, T);
        balloc(d_segStart, nSeg);
        balloc(d_segSort, nSeg);
        balloc(d_iota, T); balloc(d_perm, T); balloc(d_inv, T);
        balloc(d_keys, T); balloc(d_keys2, T);
        int perSm = 0;
        for (int f : {1, 2, 4}) {
            BCK(cudaFuncSetAttribute(batchKernel(f), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * kSmemLatWords * 4)));
            BCK(cudaFuncSetAttribute(clusterKernel(f), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * kSmemLatWords * 4)));
        }
        BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch<kInFlight>, kThreads, 2 * kSmemLatWords * 4));
        int sms = 0;
        BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu));
        grid = std::max(1, perSm) * sms;
        /* target scratch of the systems the cluster kernel may take (those
         * above 32^3 sites when the autotuner lowers the threshold) */
        if (maxLatWords > kClusterAboveLow) balloc(d_tmp, (size_t)grid * maxLatWords);
        balloc(d_clItem, (size_t)grid / 2 + 1);
        size_t bytes = 0;
        BCK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, d_keys, d_keys2, d_iota, d_perm, (int)T, 0, 64, stream));
        cubBytes = bytes;
        BCK(cudaMalloc(&d_cub, cubBytes));

        BCK(cudaMemcpyAsync(d_desc, desc.data(), S * sizeof(SysDesc), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_pos, hpos.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_img, himgRows.data(), 3 * (size_t)T * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_nbr, hnbr.data(), hnbr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_deg, hdeg.data(), T, cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_s2o, hs2o.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_lat, hlat.data(), poolWords * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_r250, hr250.data(), hr250.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_slotSeg, slotSeg.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(d_segStart, segStart.data(), nSeg * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemsetAsync(d_cnt, 0, 3 * S * sizeof(unsigned long long), stream));
        BCK(cudaMemsetAsync(d_flags, 0, T, stream));
        BCK(cudaStreamSynchronize(stream));
        pend.clear();
        pend.shrink_to_fit();
        initialized = true;
        /* the reference sorts at initialize when the age is not 0 (.cu:2511-2512) */
        std::vector<uint8_t> due(S);
        for (size_t sI = 0; sI < S; ++sI) due[sI] = age[sI] != 0;
        sortSystems(due);
    }

    /* doSpatialSorting (.cu:1835-1943) for the systems marked in due */
    void sortSystems(const std::vector<uint8_t> &due)
    {
        bool any = false;
        std::vector<uint8_t> segSort(nSeg, 0);
        for (size_t sI = 0; sI < desc.size(); ++sI)
            if (due[sI]) {
                any = true;
                for (uint32_t g = segOfSys[sI]; g < segOfSys[sI + 1]; ++g) segSort[g] = 1;
            }
        if (!any) return;
        BCK(cudaMemcpyAsync(d_segSort, segSort.data(), nSeg, cudaMemcpyHostToDevice, stream));
        const int blocks = (int)std::min<uint32_t>((T + 255) / 256, 148 * 16);
        k_sort_keys<<<blocks, 256, 0, stream>>>(d_pos, d_slotSeg, d_segStart, d_segSort, T, d_keys, d_iota);
        uint32_t segBits = 1;
        while ((1u << segBits) < nSeg) ++segBits;
        size_t bytes = cubBytes;
        BCK(cub::DeviceRadixSort::SortPairs(d_cub, bytes, d_keys, d_keys2, d_iota, d_perm, (int)T, 0, (int)(32 + segBits), stream));
        k_inv<<<blocks, 256, 0, stream>>>(d_perm, d_inv, T);
        k_perm<<<blocks, 256, 0, stream>>>(d_perm, d_inv, T, rows, d_pos, d_img, d_nbr, d_deg, d_s2o, d_pos2, d_img2, d_nbr2,
                                           d_deg2, d_s2o2);
        BCK(cudaGetLastError());
        std::swap(d_pos, d_pos2);
        std::swap(d_img, d_img2);
        std::swap(d_nbr, d_nbr2);
        std::swap(d_deg, d_deg2);
        std::swap(d_s2o, d_s2o2);
    }

    /* clusters of cs CTAs of k_batch_cl that can be resident at once (0: none) */
    int activeClusters(int cs)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)cs);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = 2 * kSmemLatWords * 4;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, clusterKernel(inFlight), &cfg) != cudaSuccess) {
            (void)cudaGetLastError();
            return 0;
        }
        return n;
    }

    /* after trial t: at the end of a stage, keep the stage's default unless
     * a candidate is more than 3% faster per attempted move (skipped trials
     * are recorded as 0 and not candidates) */
    void finishTrial(size_t t)
    {
        const std::vector<double> &ns = trialNsPerMove;
        static const int kCand[4] = {4, 2, 8, 0};
        if (t == 3) {
            size_t best = 0;
            for (size_t c = 1; c < 4; ++c)
                if (ns[c] > 0 && ns[c] < 0.97 * ns[best]) best = c;
            clusterSize = kCand[best];
            tunedNs = ns[best];
        } else if (t == 5) {
            int f = kInFlight;
            double b = tunedNs;
            if (ns[4] > 0 && ns[4] < 0.97 * b) { f = 1; b = ns[4]; }
            if (ns[5] > 0 && ns[5] < 0.97 * b) { f = 4; b = ns[5]; }
            inFlight = f;
            tunedNs = b;
        } else if (t == 6) {
            if (ns[6] > 0 && ns[6] < 0.97 * tunedNs) {
                clusterAbove = kClusterAboveLow;
                if (clusterSize == 0) clusterSize = 4;
                tunedNs = ns[6];
            }
            tuned = true;
        }
    }

    /* every system advances by mcs[s] MCS */
    void run(const uint32_t *mcs, size_t count)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        const size_t S = desc.size();
        if (count != S || !mcs) throw ArgErr("one MCS count per system is needed");
        BCK(cudaSetDevice(gpu));
        slotOfValid = false; /* re-sorts move monomers between slots */
        std::vector<uint64_t> left(mcs, mcs + S), done(S, 0);
        std::vector<Work> hw(S);
        std::vector<uint32_t> order;
        lastLaunches = 0;
        lastAttempts = 0;
        /* the autotuner's candidates (every choice gives the same
         * trajectories); a cluster-size trial only matters with systems
         * above 64^3 sites, the threshold trial with systems of 48^3..64^3 */
        static const int kCand[4] = {4, 2, 8, 0};
        bool anyBig = false, anyMid = false;
        for (const SysDesc &d : desc) {
            anyBig |= d.latWords > kSmemLatWords;
            anyMid |= d.latWords > kClusterAboveLow && d.latWords <= kSmemLatWords;
        }
        size_t trial = autotune && !tuned ? trialNsPerMove.size() : (size_t)kTrials;
        auto applies = [&](size_t t) { return t == 0 || (t < 4 ? anyBig : t < 6 ? true : anyMid); };
        BCK(cudaEventRecord(ev0, stream));
        for (;;) {
            while (trial < (size_t)kTrials && !applies(trial)) {
                trialNsPerMove.push_back(0.0); /* skipped: affects no system of this batch */
                finishTrial(trial++);
            }
            const bool trying = trial < (size_t)kTrials;
            int cs = clusterSize, IF = inFlight;
            uint32_t above = clusterAbove;
            if (trying) {
                if (trial < 4) {
                    cs = kCand[trial];
                    IF = kInFlight;
                } else if (trial < 6) {
                    IF = trial == 4 ? 1 : 4;
                } else {
                    above = kClusterAboveLow;
                    if (cs == 0) cs = 4;
                }
            }
            const int savedIF = inFlight;
            inFlight = IF; /* activeClusters() asks for this count's kernel */
            bool unlaunchable = false;
            if (cs > 0 && activeClusters(cs) == 0) {
                if (!trying) throw Err("clusters of " + std::to_string(cs) + " CTAs cannot be launched on this GPU");
                unlaunchable = true; /* the trial runs on single CTAs and is not chosen */
                cs = 0;
            }
            /* a trial launch runs an eighth of the longest pending work
             * (2 .. 50 MCS) so that its timing represents a full launch */
            uint64_t trialSteps = 2;
            if (trying) {
                uint64_t most = 0;
                for (size_t sI = 0; sI < S; ++sI)
                    if (left[sI])
                        most = std::max<uint64_t>(most, std::min<uint64_t>(left[sI], (uint64_t)(sortEvery[sI] - age[sI] % sortEvery[sI])));
                trialSteps = std::min<uint64_t>(50, std::max<uint64_t>(2, most / 8));
            }
            /* re-sort every system that starts an MCS at a sorting point (.cu:3005) */
            std::vector<uint8_t> due(S, 0);
            order.clear();
            for (size_t sI = 0; sI < S; ++sI) {
                hw[sI].age = age[sI];
                hw[sI].steps = 0;
                hw[sI].done = (uint32_t)done[sI];
                if (!left[sI]) continue;
                due[sI] = age[sI] % sortEvery[sI] == 0;
                const uint64_t toNext = (uint64_t)(sortEvery[sI] - age[sI] % sortEvery[sI]);
                hw[sI].steps = (uint32_t)std::min<uint64_t>(left[sI], std::min<uint64_t>(toNext, trying ? trialSteps : 0xFFFFFFFFull));
                order.push_back((uint32_t)sI);
            }
            if (order.empty()) break;
            sortSystems(due);
            /* longest work first */
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
                return (uint64_t)hw[a].steps * desc[a].n > (uint64_t)hw[b].steps * desc[b].n;
            });
            /* systems with a global-memory lattice go to the cluster kernel
             * (first part of the order), the others to the single-CTA kernel */
            std::vector<uint32_t> big, small;
            for (uint32_t sI : order) ((cs > 0 && desc[sI].latWords > above) ? big : small).push_back(sI);
            order = big;
            order.insert(order.end(), small.begin(), small.end());
            BCK(cudaMemcpyAsync(d_work, hw.data(), S * sizeof(Work), cudaMemcpyHostToDevice, stream));
            BCK(cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
            BCK(cudaMemsetAsync(d_next, 0, 2 * sizeof(unsigned int), stream));
            BCK(cudaEventRecord(evT0, stream));
            BCK(cudaEventRecord(evFork, stream));
            BCK(cudaStreamWaitEvent(stream2, evFork, 0));
            Arrays A{d_pos, d_img, d_nbr, d_deg, d_flags, T, d_lat, d_tmp, maxLatWords, d_r250, d_cnt};
            /* the clusters (longest work) are launched first, the single-CTA
             * kernel fills the remaining slots and those the clusters free */
            if (!big.empty()) {
                const size_t clusters = std::max<size_t>(1, std::min<size_t>((size_t)grid / (size_t)cs, big.size()));
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)(clusters * (size_t)cs));
                cfg.blockDim = dim3(kThreads);
                cfg.dynamicSmemBytes = 2 * kSmemLatWords * 4; /* distributed lattice slices */
                cfg.stream = stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = (unsigned)cs;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                const SysDesc *a0 = d_desc;
                const Work *a1 = d_work;
                const uint32_t *a2 = d_order;
                uint32_t a3 = (uint32_t)big.size();
                unsigned int *a4 = d_next;
                uint32_t *a5 = d_clItem;
                void *args[] = {&a0, &a1, &a2, &a3, &a4, &a5, &A};
                BCK(cudaLaunchKernelExC(&cfg, clusterKernel(IF), args));
                ++lastLaunches;
            }
            if (!small.empty()) {
                const int g = (int)std::min<size_t>((size_t)grid, small.size());
                const SysDesc *a0 = d_desc;
                const Work *a1 = d_work;
                const uint32_t *a2 = d_order + big.size();
                uint32_t a3 = (uint32_t)small.size();
                unsigned int *a4 = d_next + 1;
                void *args[] = {&a0, &a1, &a2, &a3, &a4, &A};
                BCK(cudaLaunchKernel(batchKernel(IF), dim3((unsigned)g), dim3(kThreads), args, 2 * kSmemLatWords * 4, stream2));
                ++lastLaunches;
            }
            inFlight = savedIF;
            BCK(cudaEventRecord(evJoin, stream2));
            BCK(cudaStreamWaitEvent(stream, evJoin, 0));
            BCK(cudaEventRecord(evT1, stream));
            /* the host buffers are reused by the next round */
            BCK(cudaStreamSynchronize(stream));
            uint64_t moves = 0;
            for (uint32_t sI : order) moves += (uint64_t)hw[sI].steps * desc[sI].n;
            if (trying) {
                float tms = 0;
                BCK(cudaEventElapsedTime(&tms, evT0, evT1));
                trialNsPerMove.push_back(unlaunchable ? 1e30 : (moves ? tms * 1e6 / (double)moves : 1e30));
                finishTrial(trial++);
            }
            for (uint32_t sI : order) {
                lastAttempts += (uint64_t)hw[sI].steps * desc[sI].n;
                age[sI] += hw[sI].steps;
                left[sI] -= hw[sI].steps;
                done[sI] += hw[sI].steps;
            }
        }
        BCK(cudaEventRecord(ev1, stream));
        BCK(cudaEventSynchronize(ev1));
        float ms = 0;
        BCK(cudaEventElapsedTime(&ms, ev0, ev1));
        lastMs = ms;
    }

    void positions(uint32_t sI, int32_t *out, size_t n)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        if (sI >= desc.size()) throw ArgErr("system index out of range");
        const SysDesc &d = desc[sI];
        if (n < d.n) throw ArgErr("output buffer too small");
        BCK(cudaSetDevice(gpu));
        if (outCap < 3 * (size_t)d.n) {
            bfree(d_out);
            balloc(d_out, 3 * (size_t)d.n);
            outCap = 3 * (size_t)d.n;
        }
        int32_t L[3];
        for (int a = 0; a < 3; ++a) L[a] = (int32_t)undilate3(d.top[a] >> a) + 1;
        const int blocks = (int)std::min<uint32_t>((d.n + 255) / 256, 148 * 8);
        k_unfold<<<blocks, 256, 0, stream>>>(d_pos, d_img, d_s2o, T, d.base, d.n, L[0], L[1], L[2], d_out);
        BCK(cudaGetLastError());
        BCK(cudaMemcpyAsync(out, d_out, 3 * (size_t)d.n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
    }

    /* unfolded positions of m selected monomers, ids[k] = (system << 32) | original id */
    void gather(const uint64_t *ids, size_t m, int32_t *out)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        if (m == 0) return;
        if (!ids || !out) throw ArgErr("ids and output are needed");
        if (m > 0xFFFFFFFFull) throw ArgErr("too many monomers in one call");
        for (size_t k = 0; k < m; ++k) {
            const uint64_t s = ids[k] >> 32, o = ids[k] & 0xFFFFFFFFull;
            if (s >= desc.size() || o >= desc[s].n) throw ArgErr("monomer id out of range at entry " + std::to_string(k));
        }
        BCK(cudaSetDevice(gpu));
        if (!d_slotOf) balloc(d_slotOf, std::max<uint32_t>(T, 1));
        if (!slotOfValid) {
            const int blocks = (int)std::min<uint32_t>((T + 255) / 256, 148 * 8);
            k_slot_of<<<std::max(blocks, 1), 256, 0, stream>>>(d_s2o, d_desc, (uint32_t)desc.size(), T, d_slotOf);
            BCK(cudaGetLastError());
            slotOfValid = true;
        }
        if (m > gCap) {
            bfree(d_gids);
            bfree(d_gout);
            balloc(d_gids, m);
            balloc(d_gout, 3 * m);
            gCap = m;
        }
        BCK(cudaMemcpyAsync(d_gids, ids, m * sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
        const int blocks = (int)std::min<size_t>((m + 255) / 256, 148 * 8);
        k_gather<<<blocks, 256, 0, stream>>>(d_pos, d_img, d_slotOf, d_desc, T, d_gids, (uint32_t)m, d_gout);
        BCK(cudaGetLastError());
        BCK(cudaMemcpyAsync(out, d_gout, 3 * m * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
    }

    /* every system's unfolded positions, systems in order, each in its original monomer order */
    void allPositions(int32_t *out, size_t n)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        if (n < T) throw ArgErr("output buffer too small");
        BCK(cudaSetDevice(gpu));
        if (outCap < 3 * (size_t)T) {
            bfree(d_out);
            balloc(d_out, 3 * (size_t)T);
            outCap = 3 * (size_t)T;
        }
        for (const SysDesc &d : desc) {
            int32_t L[3];
            for (int a = 0; a < 3; ++a) L[a] = (int32_t)undilate3(d.top[a] >> a) + 1;
            const int blocks = (int)std::min<uint32_t>((d.n + 255) / 256, 148 * 8);
            k_unfold<<<blocks, 256, 0, stream>>>(d_pos, d_img, d_s2o, T, d.base, d.n, L[0], L[1], L[2], d_out + 3 * (size_t)d.base);
        }
        BCK(cudaGetLastError());
        BCK(cudaMemcpyAsync(out, d_out, 3 * (size_t)T * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
    }

    void state(uint32_t sI, int64_t *a, uint32_t *r250, uint64_t *counters)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        if (sI >= desc.size()) throw ArgErr("system index out of range");
        BCK(cudaSetDevice(gpu));
        if (a) *a = age[sI];
        if (r250) BCK(cudaMemcpyAsync(r250, d_r250 + (size_t)sI * 251, 251 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        if (counters) BCK(cudaMemcpyAsync(counters, d_cnt + 3 * (size_t)sI, 3 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
    }

    void lattice(uint32_t sI, uint32_t *words, size_t nwords)
    {
        if (!initialized) throw Err("bfm_batch_initialize must be called first");
        if (sI >= desc.size()) throw ArgErr("system index out of range");
        if (nwords < desc[sI].latWords) throw ArgErr("output buffer too small");
        BCK(cudaSetDevice(gpu));
        BCK(cudaMemcpyAsync(words, d_lat + desc[sI].latOff, desc[sI].latWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
    }
};

} // namespace ens
} // namespace bfm

struct bfm_batch {
    bfm::ens::Batch b;
};

#define BGUARD(h, ...)                                      \
    do {                                                    \
        if (!(h)) return BFM_EINVAL;                        \
        try {                                               \
            __VA_ARGS__;                                    \
            return BFM_OK;                                  \
        } catch (bfm::ens::ArgErr const &ex) {              \
            (h)->b.err = ex.what();                         \
            return BFM_EINVAL;                              \
        } catch (bfm::ens::CudaErr const &ex) {             \
            (h)->b.err = ex.what();                         \
            return BFM_ECUDA;                               \
        } catch (std::exception const &ex) {                \
            (h)->b.err = ex.what();                         \
            return BFM_ERUNTIME;                            \
        }                                                   \
    } while (0)

extern "C" {

int bfm_batch_create(int gpu, bfm_batch **out)
{
    if (!out) return BFM_EINVAL;
    try {
        auto *h = new bfm_batch();
        h->b.gpu = gpu;
        *out = h;
        return BFM_OK;
    } catch (...) {
        return BFM_ERUNTIME;
    }
}

int bfm_batch_destroy(bfm_batch *h)
{
    if (!h) return BFM_EINVAL;
    delete h;
    return BFM_OK;
}

const char *bfm_batch_last_error(const bfm_batch *h) { return h ? h->b.err.c_str() : "null batch handle"; }

int bfm_batch_add_system(bfm_batch *h, uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, const int32_t *pos3, const uint8_t *deg,
                         const uint32_t *nbr8, const uint8_t *allowed512, int rng, int64_t age, int64_t sort_every,
                         const uint32_t *r250_state251, uint64_t r250_seed, uint32_t *sys)
{
    BGUARD(h, {
        const uint32_t L[3] = {Lx, Ly, Lz};
        const uint32_t id = h->b.add(L, n, pos3, deg, nbr8, allowed512, rng, age, sort_every, r250_state251, r250_seed);
        if (sys) *sys = id;
    });
}

int bfm_batch_initialize(bfm_batch *h) { BGUARD(h, { h->b.initialize(); }); }

int bfm_batch_set_clusters(bfm_batch *h, int size)
{
    BGUARD(h, {
        if (size != 0 && size != 1 && size != 2 && size != 4 && size != 8)
            throw bfm::ens::ArgErr("cluster size must be 0 (off), 1 (default, 4), 2, 4 or 8");
        h->b.clusterSize = size == 1 ? 4 : size;
        h->b.autotune = false;
    });
}

int bfm_batch_set_autotune(bfm_batch *h, int on)
{
    BGUARD(h, {
        h->b.autotune = on != 0;
        h->b.tuned = false;
        h->b.trialNsPerMove.clear();
        h->b.inFlight = bfm::ens::kInFlight;
        h->b.clusterAbove = bfm::ens::kSmemLatWords;
    });
}

int bfm_batch_set_shape(bfm_batch *h, int in_flight, int clusters_from_48)
{
    BGUARD(h, {
        if (in_flight != 1 && in_flight != 2 && in_flight != 4) throw bfm::ens::ArgErr("monomers in flight must be 1, 2 or 4");
        h->b.inFlight = in_flight;
        h->b.clusterAbove = clusters_from_48 ? bfm::ens::kClusterAboveLow : bfm::ens::kSmemLatWords;
        h->b.autotune = false;
    });
}

int bfm_batch_get_clusters(const bfm_batch *h, int *size, int *tuned, double *trial_ns_per_move4)
{
    if (!h) return BFM_EINVAL;
    if (size) *size = h->b.clusterSize;
    if (tuned) *tuned = h->b.tuned ? 1 : 0;
    if (trial_ns_per_move4)
        for (size_t c = 0; c < 4; ++c) trial_ns_per_move4[c] = c < h->b.trialNsPerMove.size() ? h->b.trialNsPerMove[c] : 0.0;
    return BFM_OK;
}

int bfm_batch_get_tuning(const bfm_batch *h, int *cluster_size, int *in_flight, uint32_t *cluster_above_words, int *tuned,
                         double *trial_ns_per_move7)
{
    if (!h) return BFM_EINVAL;
    const auto &b = h->b;
    if (cluster_size) *cluster_size = b.clusterSize;
    if (in_flight) *in_flight = b.inFlight;
    if (cluster_above_words) *cluster_above_words = b.clusterAbove;
    if (tuned) *tuned = b.tuned ? 1 : 0;
    if (trial_ns_per_move7)
        for (size_t c = 0; c < (size_t)bfm::ens::kTrials; ++c)
            trial_ns_per_move7[c] = c < b.trialNsPerMove.size() ? b.trialNsPerMove[c] : 0.0;
    return BFM_OK;
}

int bfm_batch_run(bfm_batch *h, const uint32_t *mcs, size_t nsys) { BGUARD(h, { h->b.run(mcs, nsys); }); }

int bfm_batch_get_positions(bfm_batch *h, uint32_t sys, int32_t *pos3, size_t n) { BGUARD(h, { h->b.positions(sys, pos3, n); }); }

int bfm_batch_get_all_positions(bfm_batch *h, int32_t *pos3, size_t n_total) { BGUARD(h, { h->b.allPositions(pos3, n_total); }); }

int bfm_batch_gather_positions(bfm_batch *h, const uint64_t *ids, size_t m, int32_t *pos3)
{
    BGUARD(h, { h->b.gather(ids, m, pos3); });
}

int bfm_batch_get_state(bfm_batch *h, uint32_t sys, int64_t *age, uint32_t *r250_state251, uint64_t *counters3)
{
    BGUARD(h, { h->b.state(sys, age, r250_state251, counters3); });
}

int bfm_batch_get_lattice(bfm_batch *h, uint32_t sys, uint32_t *words, size_t nwords, size_t *needed)
{
    BGUARD(h, {
        if (!h->b.initialized) throw bfm::ens::Err("bfm_batch_initialize must be called first");
        if (sys >= h->b.desc.size()) throw bfm::ens::ArgErr("system index out of range");
        if (needed) *needed = h->b.desc[sys].latWords;
        if (words) h->b.lattice(sys, words, nwords);
    });
}

int bfm_batch_info(const bfm_batch *h, uint32_t *nsys, uint64_t *monomers, uint32_t *nspecies_max, double *last_ms,
                   uint64_t *last_launches, uint64_t *last_attempts)
{
    if (!h) return BFM_EINVAL;
    const auto &b = h->b;
    uint32_t k = 0;
    for (const auto &d : b.desc) k = std::max(k, d.nSpecies);
    if (nsys) *nsys = b.initialized ? (uint32_t)b.desc.size() : (uint32_t)b.pend.size();
    if (monomers) *monomers = b.T;
    if (nspecies_max) *nspecies_max = k;
    if (last_ms) *last_ms = b.lastMs;
    if (last_launches) *last_launches = b.lastLaunches;
    if (last_attempts) *last_attempts = b.lastAttempts;
    return BFM_OK;
}

} /* extern "C" */
