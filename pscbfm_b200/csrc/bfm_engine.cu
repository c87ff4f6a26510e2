/*
 * bfm_engine.cu -- the colored BFM sweep on one B200 (sm_100a), behind the C
 * ABI declared in include/pscbfm_b200.h.
 *
 * Data layout in HBM (one handle):
 *   pos   uint32[npad]          Z-order code of the wrapped position, one slot
 *                               per monomer; slots grouped by colour (species)
 *                               in slabs padded to 128 slots (512 B)
 *   img   int32[3][npad]        periodic image counters (unfolded position =
 *                               wrapped + img * L), touched only on wrap moves
 *   nbr   uint32[maxdeg][npad]  neighbour slot ids, row j = j-th bond
 *   deg   uint8[npad]           bonds per monomer
 *   flags uint8[npad]           check -> perform hand-over (dir | 8)
 *   lat   uint32[L^3/32]        occupation, 1 bit per site, Z-order
 *   tmp   uint32[2][L^3/32]     bit lattice of move targets, double buffered
 *
 * One colour substep = k_check (RNG, bond test, leading-face test on lat,
 * mark target in tmp) + k_perform (leading-face test on tmp, apply), the
 * two-phase scheme of the reference's kernelSimulationScBFMCheckSpecies
 * (.cu:930-1028) and kernelSimulationScBFMPerformSpeciesAndApply
 * (.cu:1148-1190).  The colour, seed and RNG iteration of every substep are
 * drawn on the host exactly as runSimulationOnGPU does (.cu:3047-3066) and
 * uploaded as a schedule, so a whole chunk of substeps runs without the host.
 */
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfm_device.cuh"
#include "bfm_host.hpp"
#include "bfm_sweep.cuh"
#include "bfm_analyze.cuh"
#include "bfm_color.hpp"
#include "../../include/pscbfm_b200.h"

using namespace bfm;

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSlabAlign = 128;
constexpr uint32_t kNoId = 0xFFFFFFFFu;
constexpr uint32_t kChunk = 4096;       /* substeps per uploaded schedule chunk */
constexpr uint32_t kGraphSubsteps = 64; /* substeps per captured CUDA graph */
constexpr int kSweepThreads = 1024;     /* threads per CTA of the persistent kernel */
constexpr uint32_t kSweepSmemListMax = 48u * 1024u; /* candidate list bytes kept in shared memory */

struct Species {
    uint32_t off, n;
};

/* one colour substep, as drawn by the host */
struct Substep {
    uint16_t species;
    uint16_t buf;    /* temporary lattice buffer used by this substep */
    uint32_t seed;
    uint32_t iter;   /* RNG iteration = currentAge (.cu:3049), low 32 bits (all Saru uses) */
    uint32_t iterHi; /* high 32 bits, for Philox whose offset is the full 64-bit age */
};

struct Bondset {
    uint32_t forbidden[16]; /* 512 bits indexed by the interleaved bond code (zbond) */
};

struct Sys {
    uint32_t *pos;
    int32_t *img;
    const uint32_t *nbr;
    const uint8_t *deg;
    uint16_t *bcode;      /* bond codes zbond(partner, self), stored-bond path; layout bc_index */
    const uint8_t *rev;   /* for bond row j of a monomer: the row of the partner that points back */
    uint8_t *flags;
    uint32_t *lat;
    uint32_t *tmp;
    const Species *spec;
    unsigned long long *counters;
    unsigned long long *fstats; /* filter statistics per substep of a chunk (kFilters each), or null */
    int fmode;                  /* 1: counted as the reference's count kernels do; 2: the moves made */
    uint32_t fbytes;            /* Lx*Ly*Lz/8: bytes of the reference's bit-packed target lattice */
    uint32_t npad;
    uint32_t latWords;
    Geometry g;
    Bondset bonds;
};

/* Bond codes of a slot: rows 0 and 1 interleaved in one 32-bit word (row 0
 * in the low half), so that the check reads both with one load and a move
 * writes both with one store; rows j >= 2 follow as rows of npad entries. */
__host__ __device__ __forceinline__ size_t bc_index(uint32_t j, uint32_t slot, uint32_t npad)
{
    return j < 2u ? 2u * (size_t)slot + j : (size_t)j * npad + slot;
}
__device__ __forceinline__ uint32_t *bc_pair(uint16_t *bcode) { return reinterpret_cast<uint32_t *>(bcode); }
__device__ __forceinline__ const uint32_t *bc_pair(const uint16_t *bcode) { return reinterpret_cast<const uint32_t *>(bcode); }

/* Filter statistics of the reference's "Stats" mode
 * (UpdaterGPUScBFM_AB_Type.cu:1033-1097, :1192-1216, :2917-2936): moves of a
 * substep refused by the box walls, by an invalid bond, by an occupied
 * leading face (whatever the bonds), by an occupied face with valid bonds,
 * and candidates refused in the perform phase. */
constexpr int kFilters = 5;

/* warp-aggregated count of a predicate into a 64-bit counter */
__device__ __forceinline__ void count_warp(unsigned long long *c, bool pred)
{
    const unsigned int m = __ballot_sync(0xFFFFFFFFu, pred);
    if (m && (threadIdx.x & 31u) == 0) atomicAdd(c, (unsigned long long)__popc(m));
}

/* ------------------------------------------------------------- kernels */

__device__ __forceinline__ bool face_occupied(const uint32_t *__restrict__ lat, uint32_t r0, int dir, const Geometry &g)
{
    const Face f = zface(r0, dir, g);
    uint32_t any = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const uint32_t s = f.base | f.b[b] | f.c[c];
            any |= __ldg(lat + (s >> 5)) >> (s & 31u);
        }
    return any & 1u;
}

/* The tests of the reference's kernelCountFilteredCheck (.cu:1033-1097) for
 * one monomer and direction: the move leaves the box; else a bond becomes
 * invalid, and (independently) the leading face is occupied. */
__device__ __forceinline__ void filter_tests(const Sys &s, const uint32_t *forbid, uint32_t slot, uint32_t r0, int dir,
                                             bool &outside, bool &badBond, bool &front)
{
    outside = leaves_box(r0, dir, s.g);
    if (outside) return;
    const uint32_t r1 = zstep(r0, dir, s.g);
    for (uint32_t j = 0; j < s.deg[slot] && !badBond; ++j) {
        const uint32_t code = zbond(s.pos[s.nbr[(size_t)j * s.npad + slot]], r1);
        badBond = (forbid[code >> 5] >> (code & 31u)) & 1u;
    }
    front = face_occupied(s.lat, r0, dir, s.g);
}

/* Check phase of one colour substep, plus zeroing of the other temporary
 * buffer (used by the previous substep, needed clean by the next one). */
template <int RNG>
__global__ void __launch_bounds__(kThreads) k_check(Sys s, const Substep *__restrict__ sched, uint32_t k)
{
    const Substep d = sched[k];
    const Species sp = s.spec[d.species];
    __shared__ uint32_t forbid[16];
    if (threadIdx.x < 16) forbid[threadIdx.x] = s.bonds.forbidden[threadIdx.x];

    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    {
        uint4 *clr = reinterpret_cast<uint4 *>(s.tmp + (size_t)(d.buf ^ 1u) * s.latWords);
        const uint32_t n4 = s.latWords >> 2;
        for (uint32_t w = tid; w < n4; w += stride) clr[w] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();

    uint32_t *tmp = s.tmp + (size_t)d.buf * s.latWords;
    unsigned int nCand = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < sp.n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        int cand = 0;
        bool outside = false, badBond = false, front = false;
        if (i < sp.n) {
            const uint32_t slot = sp.off + i;
            const uint32_t r0 = s.pos[slot];
            const int dir = direction(draw<RNG>(d.seed, d.iter, i, d.iterHi));
            const uint32_t r1 = zstep(r0, dir, s.g);
            const uint32_t nb = s.deg[slot];
            bool ok = !leaves_box(r0, dir, s.g);
            if (ok)
                for (uint32_t j = 0; j < nb; ++j) {
                    const uint32_t q = s.pos[s.nbr[(size_t)j * s.npad + slot]];
                    const uint32_t code = zbond(q, r1);
                    if ((forbid[code >> 5] >> (code & 31u)) & 1u) {
                        ok = false;
                        break;
                    }
                }
            if (ok) ok = !face_occupied(s.lat, r0, dir, s.g);
            uint8_t f = 0;
            if (ok) {
                f = (uint8_t)(dir | 8);
                atomicOr(tmp + (r1 >> 5), 1u << (r1 & 31u));
                cand = 1;
            }
            s.flags[slot] = f;
            if (s.fstats) {
                /* the reference's count kernel draws IntHash directions whatever the RNG */
                const int dc = s.fmode == 1 ? direction(draw<RNG_INTHASH>(d.seed, d.iter, i)) : dir;
                filter_tests(s, forbid, slot, r0, dc, outside, badBond, front);
            }
        }
        if (s.fstats) {
            unsigned long long *c = s.fstats + (size_t)k * kFilters;
            count_warp(c + 0, outside);
            count_warp(c + 1, badBond);
            count_warp(c + 2, front);
            count_warp(c + 3, front && !badBond);
        }
        nCand += __syncthreads_count(cand);
    }
    if (threadIdx.x == 0 && nCand && s.counters) atomicAdd(s.counters + 0, (unsigned long long)nCand);
}

/* The reference's perform count (kernelCountFilteredPerform, .cu:1192-1216)
 * calls checkFront with its byte fetch (.cu:420-428) on the bit-packed
 * target lattice (UpdaterGPUScBFM_AB_Type.h:30): each of the nine face
 * sites' Z-order index is read as a byte index -- byte b holds the target
 * bits of sites 8b .. 8b+7 -- and indices past the lattice's Lx*Ly*Lz/8
 * bytes read zero (a linear texture of that size, .cu:2226-2240). */
__device__ __noinline__ bool front_bytes(const uint32_t *tmp, uint32_t r, int dir, const Geometry &g, uint32_t nbytes)
{
    const int ax = dir >> 1, a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;
    const uint32_t c = zstep(zstep(r, dir, g), dir, g);
    for (int u = -1; u <= 1; ++u) {
        const uint32_t cu = u == 0 ? c : zstep(c, 2 * a1 + (u > 0), g);
        for (int v = -1; v <= 1; ++v) {
            const uint32_t b = v == 0 ? cu : zstep(cu, 2 * a2 + (v > 0), g);
            if (b < nbytes && ((tmp[b >> 2] >> (8u * (b & 3u))) & 0xFFu)) return true;
        }
    }
    return false;
}

/* Perform phase: a candidate moves unless another candidate's target lies
 * in its leading face (the deterministic two-phase rule of the reference). */
__global__ void __launch_bounds__(kThreads) k_perform(Sys s, const Substep *__restrict__ sched, uint32_t k)
{
    const Substep d = sched[k];
    const Species sp = s.spec[d.species];
    const uint32_t *tmp = s.tmp + (size_t)d.buf * s.latWords;
    const uint32_t stride = gridDim.x * blockDim.x;
    unsigned int nAcc = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < sp.n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        int acc = 0;
        bool counted = false; /* filter [4] of the statistics */
        if (i < sp.n) {
            const uint32_t slot = sp.off + i;
            const uint8_t f = s.flags[slot];
            if (f & 8) {
                const uint32_t r0 = s.pos[slot];
                const int dir = f & 7;
                const bool refused = face_occupied(tmp, r0, dir, s.g);
                counted = refused;
                /* the reference counts after its perform-and-apply kernel has
                 * moved the monomer (.cu:3163-3197), with its byte fetch */
                if (s.fstats && s.fmode == 1)
                    counted = front_bytes(tmp, refused ? r0 : zstep(r0, dir, s.g), dir, s.g, s.fbytes);
                if (!refused) {
                    const uint32_t r1 = zstep(r0, dir, s.g);
                    const uint32_t w0 = r0 >> 5, w1 = r1 >> 5;
                    const uint32_t b0 = 1u << (r0 & 31u), b1 = 1u << (r1 & 31u);
                    if (w0 == w1) {
                        atomicXor(s.lat + w0, b0 | b1);
                    } else {
                        atomicXor(s.lat + w0, b0);
                        atomicXor(s.lat + w1, b1);
                    }
                    s.pos[slot] = r1;
                    const int ax = dir >> 1;
                    const bool wrapped = (dir & 1) ? ((r1 & axis_mask(s.g, ax)) == 0) : ((r0 & axis_mask(s.g, ax)) == 0);
                    if (wrapped) s.img[(size_t)ax * s.npad + slot] += (dir & 1) ? 1 : -1;
                    acc = 1;
                }
            }
        }
        if (s.fstats) count_warp(s.fstats + (size_t)k * kFilters + 4, counted);
        nAcc += __syncthreads_count(acc);
    }
    if (threadIdx.x == 0 && nAcc && s.counters) atomicAdd(s.counters + 1, (unsigned long long)nAcc);
}

/* 9-bit bond code minus / plus one unit along axis ax (per-axis modulo 8) */
__device__ __forceinline__ uint32_t bcode_dec(uint32_t c, uint32_t ax)
{
    const uint32_t m = 0x49u << ax;
    return (c & ~m) | (((c & m) - (1u << ax)) & m);
}
__device__ __forceinline__ uint32_t bcode_inc(uint32_t c, uint32_t ax)
{
    const uint32_t m = 0x49u << ax;
    return (c & ~m) | (((c | ~m) + (1u << ax)) & m);
}

/* per-axis negation modulo 8 of a 9-bit bond code: the code of the bond
 * seen from the partner */
__device__ __forceinline__ uint32_t bcode_neg(uint32_t c)
{
    return ((0u - (c & 0x049u)) & 0x049u) | ((0u - (c & 0x092u)) & 0x092u) | ((0u - (c & 0x124u)) & 0x124u);
}

/* bond code of every stored bond from the current positions */
__global__ void k_bondcodes(const uint32_t *__restrict__ pos, const uint32_t *__restrict__ nbr, const uint8_t *__restrict__ deg,
                            uint16_t *__restrict__ bcode, uint32_t npad)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x) {
        const uint32_t r = pos[i];
        for (uint32_t j = 0; j < deg[i]; ++j)
            bcode[bc_index(j, i, npad)] = (uint16_t)zbond(pos[nbr[(size_t)j * npad + i]], r);
    }
}

/* Bond modes of the persistent kernel */
enum SweepMode {
    SWEEP_GATHER = 0, /* bonds tested from the partners' positions */
    SWEEP_STORED = 1, /* bonds tested from stored codes (bond vector mod 8) */
    SWEEP_STAGED = 2, /* stored codes; a CTA's slab segments staged in shared memory by bulk copies */
    SWEEP_WINDOWED = 6 /* stored codes; independent work done inside the barrier waits (k_sweep_w), 6..8 */
};

/* k_sweep in the stored-code mode tests bonds first, on chunks of
 * kBondFirstRounds items per thread, and keeps the items that pass (index
 * and direction, position) in shared memory after the face table and the
 * candidate list: 8 B for each item of a chunk */
constexpr uint32_t kBondFirstRounds = 4;
constexpr size_t kBondFirstBytes = (size_t)kBondFirstRounds * kSweepThreads * sizeof(uint2);

/* The face-mask table in shared memory, split by word g of the face and
 * replicated kTabReplicas times (entry e, word g, copy r at
 * (g * 192 + e) * kTabReplicas + r), read by lane % kTabReplicas: lanes
 * reading different entries rarely share a bank.  48 KB. */
constexpr uint32_t kTabReplicas = 8;
constexpr size_t kWinTableBytes = (size_t)4 * 192 * kTabReplicas * 8;

__device__ __forceinline__ void build_split_table(unsigned long long *tab)
{
    for (uint32_t e = threadIdx.x; e < 192; e += blockDim.x) {
        unsigned long long m[4];
        face_table_entry((int)e, m);
        for (uint32_t g = 0; g < 4; ++g)
            for (uint32_t r = 0; r < kTabReplicas; ++r) tab[((size_t)g * 192 + e) * kTabReplicas + r] = m[g];
    }
}

/* occupied sites of a face in lattice L; which of words 1..3 it touches
 * follows from the face's spill flags (the transverse ranges spill over
 * into the next brick when their first site has low coordinate bits >= 2),
 * so the loads do not wait for the masks */
__device__ __forceinline__ unsigned long long split_occupied(const unsigned long long *L, const FaceW &fw,
                                                             const unsigned long long *tab, uint32_t lane)
{
    const bool sb = ((fw.t >> 2) & 3u) >= 2u, sc = (fw.t & 3u) >= 2u;
    const unsigned long long *tp = tab + (size_t)fw.t * kTabReplicas + (lane & (kTabReplicas - 1u));
    constexpr size_t G = (size_t)192 * kTabReplicas;
    unsigned long long o = L[fw.w[0]] & tp[0];
    if (sb) o |= L[fw.w[1]] & tp[G];
    if (sc) o |= L[fw.w[2]] & tp[2 * G];
    if (sb && sc) o |= L[fw.w[3]] & tp[3 * G];
    return o;
}

/* Shared-memory layout of the staged mode for a window of W items (W a
 * multiple of 16), after the face-mask table: positions (4 B), bond codes
 * rows 0 and 1 (one 32-bit word), bond count and direction (1 B each), then
 * the candidate list (all modes keep the table first). */
struct StageLayout {
    uint32_t W;
    __host__ __device__ size_t pos() const { return kWinTableBytes; }
    __host__ __device__ size_t bc() const { return kWinTableBytes + (size_t)W * 4; }
    __host__ __device__ size_t dg() const { return kWinTableBytes + (size_t)W * 8; }
    __host__ __device__ size_t dirs() const { return kWinTableBytes + (size_t)W * 9; }
    __host__ __device__ size_t list() const { return kWinTableBytes + (size_t)W * 10; }
    __host__ __device__ size_t bytes(uint32_t cap) const { return list() + (size_t)cap * 8; }
};

/* The persistent sweep kernel (see bfm_sweep.cuh): substeps [k0, k1) of
 * the schedule, check / barrier / perform / barrier per substep.  Each CTA
 * owns one contiguous range of every colour slab (equal work per SM, a
 * compact Z-order region per CTA). */
template <int RNG, int MODE>
__global__ void __launch_bounds__(kSweepThreads, 1)
    k_sweep(Sys s, const Substep *__restrict__ sched, uint32_t k0, uint32_t k1, GridBarrier *bar, uint2 *glist,
            uint32_t cap, unsigned long long timeoutNs, uint32_t maxdeg, uint32_t window)
{
    constexpr bool STORED = MODE != SWEEP_GATHER;
    constexpr bool STAGE = MODE == SWEEP_STAGED;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ __align__(16) DirConst s_dir[6];
    __shared__ uint32_t s_forbid[16];
    __shared__ uint32_t s_after[6 * 16]; /* forbidden after a move in dir: bit (code) of row dir */
    __shared__ unsigned int s_cnt[2];     /* candidate count of the even / odd substep */
    __shared__ __align__(8) unsigned long long s_mbar;

    const StageLayout lay{window};
    uint32_t *st_pos = reinterpret_cast<uint32_t *>(s_dyn + lay.pos());
    uint32_t *st_bc = reinterpret_cast<uint32_t *>(s_dyn + lay.bc());
    uint8_t *st_dg = s_dyn + lay.dg();
    uint8_t *st_dir = s_dyn + lay.dirs();
    uint2 *list = glist ? glist + (size_t)blockIdx.x * cap : reinterpret_cast<uint2 *>(s_dyn + (STAGE ? lay.list() : kWinTableBytes));
    unsigned long long *s_tab = reinterpret_cast<unsigned long long *>(s_dyn);
    /* stored-code mode: the items of a chunk whose bonds allow the move */
    uint2 *bondok = reinterpret_cast<uint2 *>(s_dyn + kWinTableBytes + (glist ? 0 : (size_t)cap * sizeof(uint2)));
    __shared__ unsigned int s_nok[2];
    uint32_t chunk = 0;

    build_split_table(s_tab);
    build_dir_table(s_dir, s.g);
    if (threadIdx.x < 16) s_forbid[threadIdx.x] = s.bonds.forbidden[threadIdx.x];
    if (threadIdx.x < 96) {
        const uint32_t dir = threadIdx.x >> 4, w = threadIdx.x & 15u, ax = dir >> 1;
        uint32_t bits = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint32_t c = w * 32u + b;
            const uint32_t nc = (dir & 1u) ? bcode_dec(c, ax) : bcode_inc(c, ax); /* (q - r0) - D */
            bits |= ((s.bonds.forbidden[nc >> 5] >> (nc & 31u)) & 1u) << b;
        }
        s_after[threadIdx.x] = bits;
    }
    if (threadIdx.x == 0) {
        s_cnt[0] = s_cnt[1] = 0;
        s_nok[0] = s_nok[1] = 0;
        if (STAGE) {
            mbar_init(&s_mbar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    unsigned int target = 0; /* counting barrier: arrivals expected so far */
    uint32_t mphase = 0;      /* parity of the staging mbarrier */
    __syncthreads();

    unsigned long long *lat = reinterpret_cast<unsigned long long *>(s.lat);
    unsigned long long *tmp = reinterpret_cast<unsigned long long *>(s.tmp);
    const uint32_t words = s.latWords >> 1;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t npad = s.npad;
    const uint32_t *__restrict__ nbr = s.nbr;
    const uint8_t *__restrict__ deg = s.deg;
    uint16_t *bcode = s.bcode;
    uint32_t *pos = s.pos;
    unsigned int nCand = 0, nAcc = 0;
    uint32_t prevBuf = 0;
    bool havePrev = false;
    bool alive = true;

    for (uint32_t k = k0; k < k1; ++k) {
        const Substep d = sched[k];
        const Species sp = s.spec[d.species];
        const uint32_t lo = (uint32_t)(((uint64_t)sp.n * blockIdx.x) / gridDim.x);
        const uint32_t hi = (uint32_t)(((uint64_t)sp.n * (blockIdx.x + 1)) / gridDim.x);
        const uint32_t wlo = lo & ~15u;
        unsigned int &cnt = s_cnt[k & 1u];

        if (STAGE && threadIdx.x == 0) {
            /* stage this CTA's segments of the slab: all copies in flight at once */
            const uint32_t wn = ((hi + 15u) & ~15u) - wlo;
            const uint32_t codes = maxdeg > 0 ? 4u : 0u;
            fence_proxy_async();
            mbar_arrive_expect_tx(&s_mbar, wn * (4u + 1u + codes));
            bulk_g2s(st_pos, pos + sp.off + wlo, wn * 4u, &s_mbar);
            bulk_g2s(st_dg, deg + sp.off + wlo, wn, &s_mbar);
            if (codes) bulk_g2s(st_bc, bc_pair(bcode) + sp.off + wlo, wn * 4u, &s_mbar);
        }
        /* zero the target words this CTA's candidates set in the previous substep */
        if (havePrev) {
            unsigned long long *tp = tmp + (size_t)prevBuf * words;
            const unsigned int pc = s_cnt[(k - 1u) & 1u];
            for (uint32_t j = threadIdx.x; j < pc; j += blockDim.x) {
                const uint2 e = list[j];
                const int dir = (int)(e.x >> 28);
                tp[dstep(e.y, dir, s_dir[dir]) >> 6] = 0ull;
            }
        }
        if (STAGE) {
            /* directions of all items while the copies are in flight */
            for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
                st_dir[i - wlo] = (uint8_t)direction(draw<RNG>(d.seed, d.iter, i, d.iterHi));
        }
        if (threadIdx.x == 0) cnt = 0;
        __syncthreads();
        if (STAGE) {
            if (!mbar_wait_bounded(&s_mbar, mphase, timeoutNs)) atomicExch(&bar->err, 1u);
            mphase ^= 1u;
        }

        /* phase A: check this CTA's contiguous range [lo, hi) of the slab */
        unsigned long long *tb = tmp + (size_t)d.buf * words;
        if constexpr (MODE == SWEEP_STORED) {
            /* bonds first, on chunks of kBondFirstRounds items per thread
             * (bond counts, bond codes and positions of a chunk loaded
             * together); the items that pass -- most moves of a dense melt
             * fail on their bonds -- take the leading-face test in blocks of
             * 64 per warp, a lane's two lattice probes in flight together.
             * Same candidates as the one-pass loop below, in another list
             * order, on which no result depends.  Two counters alternate
             * between chunks, so one CTA barrier per pass suffices. */
            const uint32_t T = blockDim.x, NW = T >> 5, warp = threadIdx.x >> 5, lanemask = (1u << lane) - 1u;
            for (uint32_t cb = lo; cb < hi; cb += kBondFirstRounds * T, ++chunk) {
                unsigned int &nokc = s_nok[chunk & 1u];
                if (threadIdx.x == 0) s_nok[(chunk + 1u) & 1u] = 0; /* last read before the previous chunk's end */
                uint32_t dg[kBondFirstRounds], pr[kBondFirstRounds], r0[kBondFirstRounds];
#pragma unroll
                for (uint32_t u = 0; u < kBondFirstRounds; ++u) {
                    const uint32_t ii = cb + u * T + threadIdx.x;
                    const bool live = ii < hi;
                    const uint32_t slot = sp.off + (live ? ii : lo);
                    dg[u] = live ? deg[slot] : 0u;
                    pr[u] = (live && maxdeg > 0) ? bc_pair(bcode)[slot] : 0u;
                    r0[u] = live ? pos[slot] : 0u;
                }
#pragma unroll
                for (uint32_t u = 0; u < kBondFirstRounds; ++u) {
                    const uint32_t ii = cb + u * T + threadIdx.x;
                    bool ok = ii < hi;
                    int dir = 0;
                    if (ok) {
                        dir = direction(draw<RNG>(d.seed, d.iter, ii, d.iterHi));
                        if (s.g.open) ok = !leaves_box(r0[u], dir, s.g);
                        const uint32_t *after = s_after + dir * 16;
                        const uint32_t ea = pr[u] & 0xFFFFu, eb = pr[u] >> 16;
                        if (dg[u] > 0) ok = ok && !((after[ea >> 5] >> (ea & 31u)) & 1u);
                        if (dg[u] > 1) ok = ok && !((after[eb >> 5] >> (eb & 31u)) & 1u);
                        for (uint32_t j = 2; ok && j < dg[u]; ++j) {
                            const uint32_t c = bcode[(size_t)j * npad + sp.off + ii];
                            if ((after[c >> 5] >> (c & 31u)) & 1u) ok = false;
                        }
                    }
                    const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                    unsigned int at = 0;
                    if (lane == 0 && m) at = atomicAdd(&nokc, (unsigned int)__popc(m));
                    at = __shfl_sync(0xFFFFFFFFu, at, 0);
                    if (ok) bondok[at + __popc(m & lanemask)] = make_uint2((ii - cb) | ((uint32_t)dir << 28), r0[u]);
                }
                __syncthreads();
                const uint32_t nok = nokc;
                for (uint32_t kb = warp * 64u; kb < nok; kb += 64u * NW) { /* warp-uniform */
                    uint2 e[2];
                    FaceW fw[2];
                    bool v[2];
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const uint32_t j = kb + (uint32_t)u * 32u + lane;
                        v[u] = j < nok;
                        e[u] = bondok[v[u] ? j : kb];
                        fw[u] = face_words(e[u].y, (int)(e[u].x >> 28), s.g);
                    }
                    unsigned long long occ[2];
#pragma unroll
                    for (int u = 0; u < 2; ++u) occ[u] = v[u] ? split_occupied(lat, fw[u], s_tab, lane) : 1ull;
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const bool ok = occ[u] == 0ull;
                        const int dir = (int)(e[u].x >> 28);
                        if (ok) {
                            const uint32_t r1 = dstep(e[u].y, dir, s_dir[dir]);
                            atomicOr(tb + (r1 >> 6), 1ull << (r1 & 63u));
                        }
                        const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                        if (m) {
                            const int leader = __ffs(m) - 1;
                            unsigned int at = 0;
                            if ((int)lane == leader) at = atomicAdd(&cnt, (unsigned int)__popc(m));
                            at = __shfl_sync(0xFFFFFFFFu, at, leader);
                            const uint32_t slot = sp.off + cb + (e[u].x & 0x0FFFFFFFu);
                            if (ok) list[at + __popc(m & lanemask)] = make_uint2(slot | ((uint32_t)dir << 28), e[u].y);
                        }
                        nCand += ok ? 1u : 0u;
                    }
                }
                __syncthreads();
            }
        } else {
            uint32_t i = lo + threadIdx.x;
            uint32_t nr0 = 0, ndg = 0, na = 0, nb = 0;
            if (!STAGE && i < hi) {
                const uint32_t slot = sp.off + i;
                nr0 = pos[slot];
                ndg = deg[slot];
                if (STORED) {
                    const uint32_t pr = maxdeg > 0 ? bc_pair(bcode)[slot] : 0u;
                    na = pr & 0xFFFFu;
                    nb = pr >> 16;
                } else {
                    na = maxdeg > 0 ? nbr[slot] : 0u;
                    nb = maxdeg > 1 ? nbr[(size_t)npad + slot] : 0u;
                }
            }
            for (uint32_t base = lo; base < hi; base += blockDim.x, i += blockDim.x) {
                const bool valid = i < hi;
                uint32_t r0, dg, ea, eb;
                int dir = 0;
                if (STAGE) {
                    const uint32_t w = valid ? i - wlo : 0u;
                    r0 = st_pos[w];
                    dg = st_dg[w];
                    const uint32_t pr = maxdeg > 0 ? st_bc[w] : 0u;
                    ea = pr & 0xFFFFu;
                    eb = pr >> 16;
                    dir = st_dir[w];
                } else {
                    r0 = nr0;
                    dg = ndg;
                    ea = na;
                    eb = nb;
                    const uint32_t inext = i + blockDim.x;
                    if (inext < hi) {
                        const uint32_t slot = sp.off + inext;
                        nr0 = pos[slot];
                        ndg = deg[slot];
                        if (STORED) {
                            const uint32_t pr = maxdeg > 0 ? bc_pair(bcode)[slot] : 0u;
                            na = pr & 0xFFFFu;
                            nb = pr >> 16;
                        } else {
                            na = maxdeg > 0 ? nbr[slot] : 0u;
                            nb = maxdeg > 1 ? nbr[(size_t)npad + slot] : 0u;
                        }
                    }
                }
                bool ok = false;
                if (valid) {
                    if (!STAGE) dir = direction(draw<RNG>(d.seed, d.iter, i, d.iterHi));
                    const DirConst dc = s_dir[dir];
                    const FaceW fw = face_words(r0, dir, s.g);
                    const uint32_t r1 = dstep(r0, dir, dc);
                    if (STORED) {
                        const uint32_t *after = s_after + dir * 16;
                        ok = !split_occupied(lat, fw, s_tab, lane) && !leaves_box(r0, dir, s.g);
                        if (dg > 0) ok = ok && !((after[ea >> 5] >> (ea & 31u)) & 1u);
                        if (dg > 1) ok = ok && !((after[eb >> 5] >> (eb & 31u)) & 1u);
                        for (uint32_t j = 2; j < dg; ++j) {
                            const uint32_t c = bcode[(size_t)j * npad + sp.off + i];
                            if ((after[c >> 5] >> (c & 31u)) & 1u) ok = false;
                        }
                    } else {
                        const uint32_t p0 = pos[ea];
                        const uint32_t p1 = pos[eb];
                        ok = !split_occupied(lat, fw, s_tab, lane) && !leaves_box(r0, dir, s.g);
                        if (dg > 0) {
                            const uint32_t c = zbond(p0, r1);
                            ok = ok && !((s_forbid[c >> 5] >> (c & 31u)) & 1u);
                        }
                        if (dg > 1) {
                            const uint32_t c = zbond(p1, r1);
                            ok = ok && !((s_forbid[c >> 5] >> (c & 31u)) & 1u);
                        }
                        for (uint32_t j = 2; j < dg; ++j) {
                            const uint32_t c = zbond(pos[nbr[(size_t)j * npad + sp.off + i]], r1);
                            if ((s_forbid[c >> 5] >> (c & 31u)) & 1u) ok = false;
                        }
                    }
                    if (ok) atomicOr(tb + (r1 >> 6), 1ull << (r1 & 63u));
                }
                const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                if (m) {
                    const int leader = __ffs(m) - 1;
                    unsigned int at = 0;
                    if ((int)lane == leader) at = atomicAdd(&cnt, (unsigned int)__popc(m));
                    at = __shfl_sync(0xFFFFFFFFu, at, leader);
                    if (ok) list[at + __popc(m & ((1u << lane) - 1u))] = make_uint2((sp.off + i) | ((uint32_t)dir << 28), r0);
                }
                nCand += ok ? 1u : 0u;
            }
        }
        if (!grid_barrier_count(bar, target, gridDim.x, timeoutNs)) {
            alive = false;
            break;
        }

        /* phase B: perform, this CTA's candidates only */
        {
            const unsigned long long *tr = tmp + (size_t)d.buf * words;
            const unsigned int cc = cnt;
            for (uint32_t j = threadIdx.x; j < cc; j += blockDim.x) {
                const uint2 e = list[j];
                const int dir = (int)(e.x >> 28);
                const uint32_t slot = e.x & 0x0FFFFFFFu;
                const uint32_t r0 = e.y;
                const DirConst dc = s_dir[dir];
                const FaceW fw = face_words(r0, dir, s.g);
                /* bond data of a possible move, loaded together with the probe */
                uint32_t dgm = 0, q0 = 0, q1 = 0, v0 = 0, v1 = 0, c0 = 0, c1 = 0;
                if (STORED) {
                    dgm = deg[slot];
                    if (maxdeg > 0) {
                        q0 = nbr[slot];
                        v0 = s.rev[slot];
                        const uint32_t pr = bc_pair(bcode)[slot];
                        c0 = pr & 0xFFFFu;
                        c1 = pr >> 16;
                    }
                    if (maxdeg > 1) {
                        q1 = nbr[(size_t)npad + slot];
                        v1 = s.rev[(size_t)npad + slot];
                    }
                }
                if (split_occupied(tr, fw, s_tab, lane)) continue;
                const uint32_t r1 = dstep(r0, dir, dc);
                const uint32_t w0 = r0 >> 6, w1 = r1 >> 6;
                const unsigned long long b0 = 1ull << (r0 & 63u), b1 = 1ull << (r1 & 63u);
                if (w0 == w1) {
                    atomicXor(lat + w0, b0 | b1);
                } else {
                    atomicXor(lat + w0, b0);
                    atomicXor(lat + w1, b1);
                }
                pos[slot] = r1;
                const uint32_t ax = (uint32_t)(dir >> 1);
                const bool wrapped = (dir & 1) ? ((r1 & dc.ma) == 0) : ((r0 & dc.ma) == 0);
                if (wrapped) s.img[(size_t)ax * npad + slot] += (dir & 1) ? 1 : -1;
                if (STORED) {
                    /* own bonds: (q - r0) -> (q - r1); the partner's bond back is
                     * always the per-axis negation, so it is written, not read */
                    if (dgm > 0) {
                        const uint32_t n0 = (dir & 1) ? bcode_dec(c0, ax) : bcode_inc(c0, ax);
                        const uint32_t n1 = dgm > 1 ? ((dir & 1) ? bcode_dec(c1, ax) : bcode_inc(c1, ax)) : c1;
                        bc_pair(bcode)[slot] = n0 | (n1 << 16);
                        bcode[bc_index(v0, q0, npad)] = (uint16_t)bcode_neg(n0);
                        if (dgm > 1) bcode[bc_index(v1, q1, npad)] = (uint16_t)bcode_neg(n1);
                    }
                    for (uint32_t b = 2; b < dgm; ++b) {
                        const size_t own = (size_t)b * npad + slot;
                        const uint32_t nc = (dir & 1) ? bcode_dec(bcode[own], ax) : bcode_inc(bcode[own], ax);
                        bcode[own] = (uint16_t)nc;
                        bcode[bc_index(s.rev[own], nbr[own], npad)] = (uint16_t)bcode_neg(nc);
                    }
                }
                ++nAcc;
            }
        }
        if (!grid_barrier_count(bar, target, gridDim.x, timeoutNs)) {
            alive = false;
            break;
        }
        prevBuf = d.buf;
        havePrev = true;
    }
    /* every CTA has passed the last barrier: zero the last targets so the
     * next launch starts from clean target lattices */
    if (alive && havePrev) {
        unsigned long long *tp = tmp + (size_t)prevBuf * words;
        const unsigned int pc = s_cnt[(k1 - 1u) & 1u];
        for (uint32_t j = threadIdx.x; j < pc; j += blockDim.x) {
            const uint2 e = list[j];
            const int dir = (int)(e.x >> 28);
            tp[dstep(e.y, dir, s_dir[dir]) >> 6] = 0ull;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nCand += __shfl_down_sync(0xFFFFFFFFu, nCand, o);
        nAcc += __shfl_down_sync(0xFFFFFFFFu, nAcc, o);
    }
    if (lane == 0 && s.counters) {
        if (nCand) atomicAdd(s.counters + 0, (unsigned long long)nCand);
        if (nAcc) atomicAdd(s.counters + 1, (unsigned long long)nAcc);
    }
}

/* ------------------------------------------------ windowed persistent kernel
 *
 * The same substep as k_sweep (check, grid barrier, perform, grid barrier)
 * with each grid barrier split into arrival and wait, and the wait used for
 * the work that does not depend on the other CTAs:
 *   after arriving at the check->perform barrier: zero the previous
 *     substep's targets, and fetch the bond data of this CTA's candidates
 *     into registers (a candidate's own bond codes are written only by its
 *     own CTA, and the partners' CTAs do not move during this colour);
 *   after arriving at the perform->next barrier: draw the next substep's
 *     directions into shared memory.
 * A CTA owns the same range of every colour slab for the whole launch, so
 * the positions (and bond counts) of its monomers stay in shared memory
 * from the start of the launch to its end; a move writes its new position
 * there and only the lattice and the bond codes go to global memory.  Warp 0
 * stays out of the window work so that thread 0 sees the barrier complete
 * as soon as it does.  Each warp keeps its own candidate list (ballot
 * prefix sums, no atomics); the perform phase takes the candidates of all
 * warps in one index space.  The colour ranges of the CTA live in shared
 * memory and the next schedule entry is fetched a substep ahead, so no
 * global load chain starts a substep.
 */
constexpr uint32_t kWinMaxSpecies = 32;

/* Shared memory of the windowed kernel, for at most W items of one colour
 * and P items of all colours per CTA and T threads: the face-mask table
 * split by mask (word g of the face) and replicated kTabReplicas times so
 * that lanes reading different entries rarely share a bank (48 KB),
 * positions of all the
 * CTA's monomers (4 B), direction | bonds << 3 of this substep's items
 * (1 B), bond counts of all the CTA's monomers (1 B), then two sets (this
 * substep's and the previous one's) of per-warp candidate lists of
 * seg = 32 * ceil(W / T) entries, then the items of this substep whose
 * bonds allow the move (4 B each, W). */
struct WinLayout {
    uint32_t W, T, P;
    bool bf; /* bonds-first check: the list of items whose bonds allow the move */
    __host__ __device__ uint32_t seg() const
    {
        /* a warp's candidates: 32 per round of items (one-pass check), or
         * 64 per block of the bonds-first list (W / 64 blocks over T / 32 warps) */
        const uint32_t rounds = 32u * ((W + T - 1u) / T), blocks = 64u * ((W + 2u * T - 1u) / (2u * T));
        return bf && blocks > rounds ? blocks : rounds;
    }
    __host__ __device__ size_t table() const { return 0; }
    __host__ __device__ size_t pos() const { return kWinTableBytes; }
    __host__ __device__ size_t x() const { return pos() + (size_t)P * 4; }
    __host__ __device__ size_t deg() const { return x() + W; }
    __host__ __device__ size_t lists() const { return (deg() + P + 15) & ~(size_t)15; }
    __host__ __device__ size_t bondok() const { return lists() + (size_t)2 * (T / 32u) * seg() * 8u; }
    __host__ __device__ size_t bytes() const { return bondok() + (bf ? (size_t)W * 4u : 0u); }
};

/* apply an accepted move: lattice bits, position (shared memory), image
 * counter, own bond codes and the partners' codes of the bonds back
 * (per-axis negation) */
__device__ __forceinline__ void apply_move(const Sys &s, unsigned long long *lat, uint32_t *spos, uint32_t slot, uint32_t r0,
                                           int dir, const Geometry &geo, uint32_t dgm, uint32_t q0, uint32_t v0, uint32_t c0,
                                           uint32_t q1, uint32_t v1, uint32_t c1)
{
    const uint32_t npad = s.npad;
    const uint32_t ax = (uint32_t)(dir >> 1);
    const uint32_t ma = axis_mask(geo, (int)ax), ua = 1u << ax;
    const uint32_t r1 = (dir & 1) ? zinc(r0, ma, ua) : zdec(r0, ma, ua);
    const uint32_t w0 = r0 >> 6, w1 = r1 >> 6;
    const unsigned long long b0 = 1ull << (r0 & 63u), b1 = 1ull << (r1 & 63u);
    if (w0 == w1) {
        atomicXor(lat + w0, b0 | b1);
    } else {
        atomicXor(lat + w0, b0);
        atomicXor(lat + w1, b1);
    }
    *spos = r1;
    const bool wrapped = (dir & 1) ? ((r1 & ma) == 0) : ((r0 & ma) == 0);
    if (wrapped) s.img[(size_t)ax * npad + slot] += (dir & 1) ? 1 : -1;
    uint16_t *bcode = s.bcode;
    if (dgm > 0) {
        const uint32_t n0 = (dir & 1) ? bcode_dec(c0, ax) : bcode_inc(c0, ax);
        const uint32_t n1 = dgm > 1 ? ((dir & 1) ? bcode_dec(c1, ax) : bcode_inc(c1, ax)) : c1;
        bc_pair(bcode)[slot] = n0 | (n1 << 16);
        bcode[bc_index(v0, q0, npad)] = (uint16_t)bcode_neg(n0);
        if (dgm > 1) bcode[bc_index(v1, q1, npad)] = (uint16_t)bcode_neg(n1);
    }
    for (uint32_t b = 2; b < dgm; ++b) {
        const size_t own = (size_t)b * npad + slot;
        const uint32_t nc = (dir & 1) ? bcode_dec(bcode[own], ax) : bcode_inc(bcode[own], ax);
        bcode[own] = (uint16_t)nc;
        bcode[bc_index(s.rev[own], s.nbr[own], npad)] = (uint16_t)bcode_neg(nc);
    }
}

/* The two synchronisations of a substep, split into arrival and wait: the
 * counting grid barrier over all CTAs of the cooperative launch, or -- when
 * the whole launch is one thread-block cluster (CL, small systems) -- the
 * hardware cluster barrier, where every thread arrives with release and
 * waits with acquire semantics at cluster scope (which orders the global
 * lattice, target and bond-code updates between the cluster's CTAs) and a
 * CTA barrier then ends the window work. */
template <bool CL>
__device__ __forceinline__ void win_arrive(GridBarrier *bar, unsigned int &target)
{
    if (CL) asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    else grid_arrive(bar, target, gridDim.x);
}
template <bool CL>
__device__ __forceinline__ bool win_wait(GridBarrier *bar, unsigned int target, unsigned long long timeoutNs)
{
    if (CL) {
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
        __syncthreads();
        return true;
    }
    return grid_wait(bar, target, timeoutNs);
}

/* one shape of the windowed kernel: U items per thread in flight in the
 * check phase; blockDim.x threads (a multiple of 32, 64 to 1024); CL: the
 * grid is one cluster (cluster barriers instead of grid barriers); BF: the
 * check tests the bonds of every item first and the leading face only of
 * the items that pass (otherwise face and bonds together, item by item) */
template <int RNG, int U, bool CL = false, bool BF = false>
__global__ void __launch_bounds__(1024, 1)
    k_sweep_w(Sys s, const Substep *__restrict__ sched, uint32_t k0, uint32_t k1, GridBarrier *bar,
              unsigned long long timeoutNs, uint32_t maxdeg, uint32_t window, uint32_t nspec, uint32_t ptotal)
{
    const uint32_t T = blockDim.x, NW = T >> 5;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ uint32_t s_after[6 * 16];
    __shared__ uint32_t s_lo[kWinMaxSpecies], s_n[kWinMaxSpecies], s_off[kWinMaxSpecies], s_base[kWinMaxSpecies];
    __shared__ unsigned int s_wcnt[2][32];

    const WinLayout lay{window, T, ptotal, BF};
    const uint32_t seg = lay.seg();
    unsigned long long *s_tab = reinterpret_cast<unsigned long long *>(s_dyn + lay.table());
    uint32_t *spos = reinterpret_cast<uint32_t *>(s_dyn + lay.pos());
    uint8_t *px = s_dyn + lay.x();
    uint8_t *sdeg = s_dyn + lay.deg();
    uint2 *lists = reinterpret_cast<uint2 *>(s_dyn + lay.lists());
    uint32_t *bondok = reinterpret_cast<uint32_t *>(s_dyn + lay.bondok());
    __shared__ unsigned int s_nok[2];

    build_split_table(s_tab);
    for (uint32_t e = threadIdx.x; e < 96; e += T) { /* the CTA may have fewer than 96 threads */
        const uint32_t dir = e >> 4, w = e & 15u, ax = dir >> 1;
        uint32_t bits = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint32_t c = w * 32u + b;
            const uint32_t nc = (dir & 1u) ? bcode_dec(c, ax) : bcode_inc(c, ax); /* (q - r0) - D */
            bits |= ((s.bonds.forbidden[nc >> 5] >> (nc & 31u)) & 1u) << b;
        }
        s_after[e] = bits;
    }
    if (threadIdx.x < nspec) {
        /* this CTA's contiguous range of every colour slab */
        const Species sp = s.spec[threadIdx.x];
        const uint32_t lo = (uint32_t)(((uint64_t)sp.n * blockIdx.x) / gridDim.x);
        const uint32_t hi = (uint32_t)(((uint64_t)sp.n * (blockIdx.x + 1)) / gridDim.x);
        s_lo[threadIdx.x] = lo;
        s_n[threadIdx.x] = hi - lo;
        s_off[threadIdx.x] = sp.off + lo;
    }
    if (threadIdx.x < 64) s_wcnt[threadIdx.x >> 5][threadIdx.x & 31u] = 0;
    if (threadIdx.x < 2) s_nok[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t b = 0;
        for (uint32_t c = 0; c < nspec; ++c) {
            s_base[c] = b;
            b += s_n[c];
        }
    }
    __syncthreads();
    /* the CTA's positions and bond counts, resident for the launch */
    for (uint32_t c = 0; c < nspec; ++c)
        for (uint32_t w = threadIdx.x; w < s_n[c]; w += T) {
            spos[s_base[c] + w] = s.pos[s_off[c] + w];
            sdeg[s_base[c] + w] = s.deg[s_off[c] + w];
        }
    __syncthreads();

    unsigned long long *lat = reinterpret_cast<unsigned long long *>(s.lat);
    unsigned long long *tmp = reinterpret_cast<unsigned long long *>(s.tmp);
    const Geometry geo = s.g;
    const uint32_t words = s.latWords >> 1;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lanemask = (1u << lane) - 1u;
    const uint32_t npad = s.npad;
    const uint32_t *__restrict__ nbr = s.nbr;
    const uint16_t *bcode = s.bcode;
    unsigned int nCand = 0, nAcc = 0;
    unsigned int target = 0;
    bool alive = true;

    /* directions of the items of substep dn, by warps 1.. */
    auto prep = [&](const Substep &dn) {
        const uint32_t plo = s_lo[dn.species], n = s_n[dn.species], base = s_base[dn.species];
#pragma unroll 2
        for (uint32_t w = threadIdx.x - 32u; w < n; w += T - 32u)
            px[w] = (uint8_t)((uint32_t)direction(draw<RNG>(dn.seed, dn.iter, plo + w, dn.iterHi)) | ((uint32_t)sdeg[base + w] << 3));
    };
    /* zero the target words of warp wi's candidates of the substep using buffer buf, list set p */
    auto clear_targets = [&](uint32_t buf, uint32_t p, uint32_t wi) {
        unsigned long long *tp = tmp + (size_t)buf * words;
        const uint2 *pl = lists + ((size_t)p * NW + wi) * seg;
        const unsigned int pc = s_wcnt[p][wi];
        for (uint32_t j = lane; j < pc; j += 32u) {
            const uint2 e = pl[j];
            tp[zstep(e.y, (int)(e.x >> 28), geo) >> 6] = 0ull;
        }
    };
    auto occupied = [&](const unsigned long long *L, const FaceW &fw) -> unsigned long long {
        return split_occupied(L, fw, s_tab, lane);
    };

    Substep d = sched[k0];
    if (threadIdx.x >= 32) prep(d);
    __syncthreads();
    uint32_t prevBuf = 0;

    for (uint32_t k = k0; k < k1; ++k) {
        const Substep dnext = k + 1u < k1 ? sched[k + 1u] : d; /* arrives long before it is used */
        const uint32_t n = s_n[d.species], off = s_off[d.species], base = s_base[d.species];
        const uint32_t p = k & 1u;
        uint2 *wlist = lists + ((size_t)p * NW + warp) * seg;
        unsigned long long *tb = tmp + (size_t)d.buf * words;
        unsigned int wc = 0; /* this warp's candidates (warp-uniform) */
        if constexpr (BF) {
            if (threadIdx.x == 0) s_nok[p ^ 1u] = 0; /* the next substep's count (last read a substep ago) */

            /* phase A, pass 1: the bonds (and walls) of every item, U items per
             * thread at a time.  In a dense melt most moves already fail here
             * (about 70 % at volume fraction 0.5), so the items that pass are
             * gathered into one CTA-wide list (a shared-memory atomic per warp
             * and round) and only they take the leading-face test of pass 2,
             * in full warps.  The candidates are the same items as with the
             * face tested first; only their order in the lists differs, which
             * no result depends on. */
            for (uint32_t b0 = 0; b0 < n; b0 += (uint32_t)U * T) {
                uint32_t x[U], ca[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t w = b0 + (uint32_t)u * T + threadIdx.x;
                    x[u] = px[w < n ? w : 0u];
                    ca[u] = (maxdeg > 0 && w < n) ? bc_pair(bcode)[off + w] : 0u;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t w = b0 + (uint32_t)u * T + threadIdx.x;
                    const int dir = (int)(x[u] & 7u);
                    const uint32_t dg = x[u] >> 3;
                    bool ok = w < n;
                    if (ok && geo.open) ok = !leaves_box(spos[base + w], dir, geo);
                    if (ok) {
                        const uint32_t *after = s_after + dir * 16;
                        const uint32_t a0 = ca[u] & 0x1FFu, a1 = (ca[u] >> 16) & 0x1FFu;
                        if (dg > 0) ok = !((after[a0 >> 5] >> (a0 & 31u)) & 1u);
                        if (dg > 1) ok = ok && !((after[a1 >> 5] >> (a1 & 31u)) & 1u);
                        for (uint32_t j = 2; ok && j < dg; ++j) {
                            const uint32_t c = bcode[(size_t)j * npad + off + w];
                            if ((after[c >> 5] >> (c & 31u)) & 1u) ok = false;
                        }
                    }
                    const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                    unsigned int at = 0;
                    if (lane == 0 && m) at = atomicAdd(&s_nok[p], (unsigned int)__popc(m));
                    at = __shfl_sync(0xFFFFFFFFu, at, 0);
                    if (ok) bondok[at + __popc(m & lanemask)] = w | ((uint32_t)dir << 28);
                }
            }
            __syncthreads();
            /* pass 2: the leading face of the items that passed, in blocks of
             * 64 per warp, a lane's two items with their lattice loads in
             * flight together (one L2 round trip per block) */
            const uint32_t nok = s_nok[p];
            for (uint32_t cb = warp * 64u; cb < nok; cb += 64u * NW) { /* warp-uniform */
                uint32_t e[2], r0[2];
                FaceW f[2];
                bool v[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const uint32_t j = cb + (uint32_t)u * 32u + lane;
                    v[u] = j < nok;
                    e[u] = bondok[v[u] ? j : cb];
                    r0[u] = spos[base + (e[u] & 0x0FFFFFFFu)];
                    f[u] = face_words(r0[u], (int)(e[u] >> 28), geo);
                }
                unsigned long long occ[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) occ[u] = v[u] ? occupied(lat, f[u]) : 1ull;
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const bool ok = occ[u] == 0ull;
                    if (ok) {
                        const int dir = (int)(e[u] >> 28);
                        const uint32_t r1 = (dir & 1) ? zinc(r0[u], f[u].ma, f[u].ua) : zdec(r0[u], f[u].ma, f[u].ua);
                        atomicOr(tb + (r1 >> 6), 1ull << (r1 & 63u));
                    }
                    const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                    if (ok) wlist[wc + __popc(m & lanemask)] = make_uint2(e[u], r0[u]);
                    wc += __popc(m);
                }
            }
        } else {
            /* phase A: U items per thread at a time, face and bonds together */
            for (uint32_t b0 = 0; b0 < n; b0 += (uint32_t)U * T) {
                FaceW f[U];
                uint32_t r0[U], x[U], ca[U];
                unsigned long long occ[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t w = b0 + (uint32_t)u * T + threadIdx.x;
                    const uint32_t ws = w < n ? w : 0u;
                    r0[u] = spos[base + ws];
                    x[u] = px[ws];
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t w = b0 + (uint32_t)u * T + threadIdx.x;
                    f[u] = face_words(r0[u], (int)(x[u] & 7u), geo);
                    occ[u] = 1ull;
                    ca[u] = 0u;
                    if (w < n) {
                        occ[u] = occupied(lat, f[u]);
                        if (maxdeg > 0) ca[u] = bc_pair(bcode)[off + w];
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t w = b0 + (uint32_t)u * T + threadIdx.x;
                    const int dir = (int)(x[u] & 7u);
                    const uint32_t dg = x[u] >> 3;
                    bool ok = occ[u] == 0ull && !leaves_box(r0[u], dir, geo);
                    if (ok) {
                        const uint32_t *after = s_after + dir * 16;
                        const uint32_t a0 = ca[u] & 0x1FFu, a1 = (ca[u] >> 16) & 0x1FFu;
                        if (dg > 0) ok = !((after[a0 >> 5] >> (a0 & 31u)) & 1u);
                        if (dg > 1) ok = ok && !((after[a1 >> 5] >> (a1 & 31u)) & 1u);
                        for (uint32_t j = 2; ok && j < dg; ++j) {
                            const uint32_t c = bcode[(size_t)j * npad + off + w];
                            if ((after[c >> 5] >> (c & 31u)) & 1u) ok = false;
                        }
                    }
                    if (ok) {
                        const uint32_t r1 = (dir & 1) ? zinc(r0[u], f[u].ma, f[u].ua) : zdec(r0[u], f[u].ma, f[u].ua);
                        atomicOr(tb + (r1 >> 6), 1ull << (r1 & 63u));
                    }
                    const unsigned int m = __ballot_sync(0xFFFFFFFFu, ok);
                    if (ok) wlist[wc + __popc(m & lanemask)] = make_uint2(w | ((uint32_t)dir << 28), r0[u]);
                    wc += __popc(m);
                }
            }
        }
        if (lane == 0) s_wcnt[p][warp] = wc;
        nCand += lane == 0 ? wc : 0u;

        /* check -> perform barrier */
        __syncthreads();
        win_arrive<CL>(bar, target);
        /* the previous substep's targets (nobody reads or writes that buffer
         * until every CTA has passed the next barrier); warp 1 also takes
         * warp 0's */
        if (k > k0 && warp > 0) {
            clear_targets(prevBuf, p ^ 1u, warp);
            if (warp == 1) clear_targets(prevBuf, p ^ 1u, 0);
        }
        /* The CTA's candidates in one index space: lane l of every warp
         * holds the exclusive offset of warp l's list.  Candidate j goes to
         * thread 32 + j (warp 0 stays free to watch the barrier); its bond
         * data are fetched now. */
        const unsigned int cntl = lane < NW ? s_wcnt[p][lane] : 0u;
        unsigned int incl = cntl;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o) incl += t;
        }
        const unsigned int excl = incl - cntl;
        const unsigned int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        /* list entry of candidate j: the last warp whose offset is <= j */
        auto entry = [&](uint32_t j) -> uint2 {
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1) {
                const uint32_t mid = lo + step;
                const unsigned int om = __shfl_sync(0xFFFFFFFFu, excl, mid & 31u);
                if (mid < NW && om <= j) lo = mid;
            }
            return lists[((size_t)p * NW + lo) * seg + (j - __shfl_sync(0xFFFFFFFFu, excl, lo))];
        };
        const uint32_t jb = threadIdx.x - 32u;
        const bool bval = threadIdx.x >= 32 && jb < total;
        uint2 e0 = make_uint2(0u, 0u);
        uint32_t bdg = 0, bq0 = 0, bv0 = 0, bc0 = 0, bq1 = 0, bv1 = 0, bc1 = 0;
        if (warp > 0 && 32u * (warp - 1u) < total) { /* warp-uniform */
            e0 = entry(bval ? jb : 0u);
            if (bval) {
                const uint32_t w = e0.x & 0x0FFFFFFFu, slot = off + w;
                bdg = sdeg[base + w];
                if (maxdeg > 0) {
                    bq0 = nbr[slot];
                    bv0 = s.rev[slot];
                    const uint32_t pr = bc_pair(bcode)[slot];
                    bc0 = pr & 0xFFFFu;
                    bc1 = pr >> 16;
                }
                if (maxdeg > 1) {
                    bq1 = nbr[(size_t)npad + slot];
                    bv1 = s.rev[(size_t)npad + slot];
                }
            }
        }
        if (!win_wait<CL>(bar, target, timeoutNs)) {
            alive = false;
            break;
        }

        /* phase B: perform the candidates */
        {
            const unsigned long long *tr = tmp + (size_t)d.buf * words;
            if (bval) {
                const uint32_t w = e0.x & 0x0FFFFFFFu;
                if (!occupied(tr, face_words(e0.y, (int)(e0.x >> 28), geo))) {
                    apply_move(s, lat, spos + base + w, off + w, e0.y, (int)(e0.x >> 28), geo, bdg, bq0, bv0, bc0, bq1, bv1, bc1);
                    ++nAcc;
                }
            }
            for (uint32_t j0 = T - 32u; j0 < total; j0 += T) {
                /* beyond the first T - 32 candidates: all threads, fetched now */
                const uint32_t j = j0 + threadIdx.x;
                const uint2 e = entry(j < total ? j : 0u);
                if (j >= total) continue;
                const uint32_t w = e.x & 0x0FFFFFFFu, slot = off + w;
                const uint32_t dgm = sdeg[base + w];
                uint32_t q0 = 0, v0 = 0, c0 = 0, q1 = 0, v1 = 0, c1 = 0;
                if (maxdeg > 0) {
                    q0 = nbr[slot];
                    v0 = s.rev[slot];
                    const uint32_t pr = bc_pair(bcode)[slot];
                    c0 = pr & 0xFFFFu;
                    c1 = pr >> 16;
                }
                if (maxdeg > 1) {
                    q1 = nbr[(size_t)npad + slot];
                    v1 = s.rev[(size_t)npad + slot];
                }
                if (occupied(tr, face_words(e.y, (int)(e.x >> 28), geo))) continue;
                apply_move(s, lat, spos + base + w, slot, e.y, (int)(e.x >> 28), geo, dgm, q0, v0, c0, q1, v1, c1);
                ++nAcc;
            }
        }

        /* perform -> next check barrier */
        __syncthreads();
        win_arrive<CL>(bar, target);
        if (k + 1u < k1 && threadIdx.x >= 32) prep(dnext);
        if (!win_wait<CL>(bar, target, timeoutNs)) {
            alive = false;
            break;
        }
        prevBuf = d.buf;
        d = dnext;
    }
    /* every CTA has passed the last barrier: zero the last targets so the
     * next launch starts from clean target lattices */
    if (alive && k1 > k0) clear_targets(prevBuf, (k1 - 1u) & 1u, warp);
    /* positions back to global memory */
    __syncthreads();
    for (uint32_t c = 0; c < nspec; ++c)
        for (uint32_t w = threadIdx.x; w < s_n[c]; w += T) s.pos[s_off[c] + w] = spos[s_base[c] + w];
    for (int o = 16; o > 0; o >>= 1) nAcc += __shfl_down_sync(0xFFFFFFFFu, nAcc, o);
    if (lane == 0 && s.counters) {
        if (nCand) atomicAdd(s.counters + 0, (unsigned long long)nCand);
        if (nAcc) atomicAdd(s.counters + 1, (unsigned long long)nAcc);
    }
}

/* the windowed shapes: items in flight per thread in the check phase; the
 * CTA size is chosen at configuration to pack the CTA's items tightly */
constexpr int kWinU[5] = {1, 2, 4, 2, 2};
/* windowed variants 3 and 4 (shapes 9, 10): the launch is one cluster of
 * 8 or 16 CTAs, for systems small enough that each CTA holds few monomers */
constexpr int kWinCluster[5] = {0, 0, 0, 8, 16};
/* variant 2 (shape 8) tests bonds first and the face of the items that pass */
constexpr bool kWinBondFirst[5] = {false, false, true, false, false};
/* the automatic shape: variant 2 once a CTA holds this many items of a
 * colour (dense large systems, where most moves fail on their bonds and the
 * face tests saved outweigh the extra pass), variant 1 below */
constexpr uint32_t kWinBondFirstItems = 2048;

template <int RNG>
const void *win_kernel(int i)
{
    return i == 0   ? (const void *)k_sweep_w<RNG, 1>
           : i == 1 ? (const void *)k_sweep_w<RNG, 2>
           : i == 2 ? (const void *)k_sweep_w<RNG, 4, false, true>
                    : (const void *)k_sweep_w<RNG, 2, true>;
}

/* rounds grid barriers expecting `expected` CTAs; with expected > gridDim.x
 * no barrier can complete and every wait runs into its bound */
__global__ void k_barrier_selftest(GridBarrier *bar, unsigned int expected, unsigned long long timeoutNs, unsigned int rounds,
                                   int counting)
{
    unsigned int gen = 0;
    if (threadIdx.x == 0) gen = counting ? 0u : ld_acquire_gpu(&bar->gen);
    for (unsigned int r = 0; r < rounds; ++r) {
        const bool ok = counting ? grid_barrier_count(bar, gen, expected, timeoutNs) : grid_barrier(bar, expected, gen, timeoutNs);
        if (!ok) return;
    }
}

/* spatial re-sort support: inv[perm[i]] = i */
__global__ void k_invert(const uint32_t *__restrict__ perm, uint32_t *__restrict__ inv, uint32_t npad)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x) inv[perm[i]] = i;
}

/* gather every per-slot array into the new slot order and remap neighbour ids */
__global__ void k_permute(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ inv, uint32_t npad,
                          uint32_t maxdeg, const uint32_t *__restrict__ pos, const int32_t *__restrict__ img,
                          const uint32_t *__restrict__ nbr, const uint8_t *__restrict__ deg,
                          const uint32_t *__restrict__ s2o, const uint8_t *__restrict__ rev,
                          uint32_t *__restrict__ pos2, int32_t *__restrict__ img2, uint32_t *__restrict__ nbr2,
                          uint8_t *__restrict__ deg2, uint32_t *__restrict__ s2o2, uint8_t *__restrict__ rev2,
                          uint32_t *__restrict__ o2s)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x) {
        const uint32_t p = perm[i];
        pos2[i] = pos[p];
        img2[i] = img[p];
        img2[npad + i] = img[npad + p];
        img2[2 * (size_t)npad + i] = img[2 * (size_t)npad + p];
        const uint8_t dg = deg[p];
        deg2[i] = dg;
        for (uint32_t j = 0; j < maxdeg; ++j) {
            nbr2[(size_t)j * npad + i] = j < dg ? inv[nbr[(size_t)j * npad + p]] : 0u;
            rev2[(size_t)j * npad + i] = rev[(size_t)j * npad + p];
        }
        const uint32_t o = s2o[p];
        s2o2[i] = o;
        if (o != kNoId) o2s[o] = i;
    }
}

/* unfolded positions in original monomer order (doCopyBack, .cu:3402-3484) */
__global__ void k_unpack(const uint32_t *__restrict__ pos, const int32_t *__restrict__ img,
                         const uint32_t *__restrict__ s2o, uint32_t npad, int32_t Lx, int32_t Ly, int32_t Lz,
                         int32_t *__restrict__ out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x) {
        const uint32_t o = s2o[i];
        if (o == kNoId) continue;
        const uint32_t c = pos[i];
        out[3 * (size_t)o + 0] = (int32_t)undilate3(c) + img[i] * Lx;
        out[3 * (size_t)o + 1] = (int32_t)undilate3(c >> 1) + img[npad + i] * Ly;
        out[3 * (size_t)o + 2] = (int32_t)undilate3(c >> 2) + img[2 * (size_t)npad + i] * Lz;
    }
}

/* ------------------------------------------------------------- host side */

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct DeviceTimeout : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

/* The dynamic shared-memory limit of a kernel is an attribute of the
 * function on a device, shared by every handle of the process; handles
 * configured for different system sizes would otherwise lower each
 * other's limit below what their own launches request.  It is only ever
 * raised. */
void raise_smem_limit(const void *fn, size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> limit;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = limit[{dev, fn}];
    if (bytes > cur) {
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        cur = bytes;
    }
}

template <typename T>
void dalloc(T *&p, size_t n)
{
    p = nullptr;
    if (n) CK(cudaMalloc((void **)&p, n * sizeof(T)));
}
template <typename T>
void dfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

std::mutex g_r250_mutex;
R250 &global_r250()
{
    static R250 r = [] {
        R250 t;
        t.seed_u64(0);
        return t;
    }();
    return r;
}

uint32_t ilog2(uint64_t v)
{
    uint32_t l = 0;
    while (v >>= 1) ++l;
    return l;
}

struct Engine {
    /* ---- configuration (setters) */
    int gpu = 0;
    uint8_t forbidden[512]; /* linear index (dx&7)|(dy&7)<<3|(dz&7)<<6, as copyBondSet (.cu:2540-2545) */
    bool nSet = false;
    uint32_t n = 0;
    std::vector<int32_t> xyz;
    std::vector<int32_t> attr;
    std::vector<uint8_t> deg;
    std::vector<uint32_t> nbr; /* n x 8 original ids */
    uint64_t L[3] = {0, 0, 0};
    bool periodic[3] = {true, true, true};
    int64_t age = 0;
    int rng = BFM_RNG_INTHASH; /* the reference's default (.cu:1407) */
    int64_t sortEvery = 5000;
    int launchMode = 0;
    int coloringMode = 0; /* 0 host walk (the reference's); 1 device for forests, host otherwise */
    int filterStats = 0; /* the reference's "Stats" filter analysis: 0 off, 1 counted as the reference, 2 the moves made */

    /* ---- derived at initialize */
    int colorOnDevice = 0; /* last initialize: 0 host walk, 1 device, 2 device for the tree components */
    bool initialized = false;
    Geometry g{};
    Bondset bonds{};
    uint32_t Lm = 0, keyBits = 0;
    size_t latWords = 0;
    std::vector<uint32_t> color;
    std::vector<Species> spec;
    uint32_t nSpecies = 0, npad = 0, maxdeg = 0, nmax = 0;

    /* ---- device state */
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t *d_pos = nullptr, *d_pos2 = nullptr;
    int32_t *d_img = nullptr, *d_img2 = nullptr;
    uint32_t *d_nbr = nullptr, *d_nbr2 = nullptr;
    uint8_t *d_deg = nullptr, *d_deg2 = nullptr;
    uint8_t *d_rev = nullptr, *d_rev2 = nullptr;
    uint16_t *d_bcode = nullptr;
    bool storedBonds = false; /* every bond has a partner entry pointing back */
    uint32_t *d_s2o = nullptr, *d_s2o2 = nullptr, *d_o2s = nullptr;
    uint8_t *d_flags = nullptr;
    uint32_t *d_lat = nullptr, *d_tmp = nullptr;
    Species *d_spec = nullptr;
    Substep *d_sched[2] = {nullptr, nullptr};
    Substep *h_sched[2] = {nullptr, nullptr};
    cudaEvent_t schedFree[2] = {nullptr, nullptr};
    unsigned long long *d_counters = nullptr;
    uint32_t *d_perm = nullptr, *d_inv = nullptr, *d_iota = nullptr, *d_keys = nullptr;
    void *d_cub = nullptr;
    size_t cubBytes = 0;
    int32_t *d_out = nullptr;
    int32_t *h_out = nullptr;
    unsigned int *h_flag = nullptr;
    bool hostPosValid = false;

    /* persistent kernel */
    GridBarrier *d_bar = nullptr;
    uint2 *d_glist = nullptr;
    int sweepGrid = 0;
    uint32_t sweepCap = 0;
    size_t sweepSmem = 0;
    unsigned long long timeoutNs = 2000000000ull;

    /* graphs: [schedule buffer][rng kind index] */
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graphRng = -1;

    uint64_t substepCounter = 0;
    uint64_t nAttempts = 0;
    bool sortedFresh = false;
    double lastRunMs = 0;
    uint64_t lastLaunches = 0;

    std::string err;

    ~Engine() { release(); }

    void requireN(uint32_t i) const
    {
        if (!nSet) throw std::runtime_error("setNrOfAllMonomers has not been called");
        if (i >= n) throw InvalidArgument("monomer index " + std::to_string(i) + " out of range (n = " + std::to_string(n) + ")");
    }

    void release()
    {
        if (stream) cudaStreamSynchronize(stream);
        for (auto &ge : graph)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
        graphRng = -1;
        dfree(d_pos); dfree(d_pos2); dfree(d_img); dfree(d_img2); dfree(d_nbr); dfree(d_nbr2);
        dfree(d_deg); dfree(d_deg2); dfree(d_rev); dfree(d_rev2); dfree(d_bcode); dfree(d_s2o); dfree(d_s2o2); dfree(d_o2s); dfree(d_flags);
        dfree(d_lat); dfree(d_tmp); dfree(d_spec); dfree(d_counters); dfree(d_perm); dfree(d_inv);
        dfree(d_iota); dfree(d_keys); dfree(d_out); dfree(d_bar); dfree(d_glist); dfree(d_fstats);
        fcnt.clear();
        releaseAnalyzer();
        if (d_cub) cudaFree(d_cub);
        d_cub = nullptr;
        for (int b = 0; b < 2; ++b) {
            dfree(d_sched[b]);
            if (h_sched[b]) cudaFreeHost(h_sched[b]);
            h_sched[b] = nullptr;
            if (schedFree[b]) cudaEventDestroy(schedFree[b]);
            schedFree[b] = nullptr;
        }
        if (h_out) cudaFreeHost(h_out);
        h_out = nullptr;
        if (h_flag) cudaFreeHost(h_flag);
        h_flag = nullptr;
        for (auto e : profEvents) cudaEventDestroy(e);
        profEvents.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        ev0 = ev1 = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        initialized = false;
        hostPosValid = false;
    }

    Sys sys() const
    {
        Sys s;
        s.pos = d_pos;
        s.img = d_img;
        s.nbr = d_nbr;
        s.deg = d_deg;
        s.bcode = d_bcode;
        s.rev = d_rev;
        s.flags = d_flags;
        s.lat = d_lat;
        s.tmp = d_tmp;
        s.spec = d_spec;
        s.counters = d_counters;
        s.fstats = filterStats ? d_fstats : nullptr;
        s.fmode = filterStats;
        s.fbytes = (uint32_t)(L[0] * L[1] * L[2] / 8);
        s.npad = npad;
        s.latWords = (uint32_t)latWords;
        s.g = g;
        s.bonds = bonds;
        return s;
    }

    /* ------------------------------------------------------ initialize */
    void initialize()
    {
        if (initialized)
            throw std::runtime_error("Initialize was already called and may not be called again until cleanup was called!");
        if (!nSet || n == 0) throw std::runtime_error("setNrOfAllMonomers must be called with n > 0 before initialize");
        for (int a = 0; a < 3; ++a)
            if (L[a] == 0) throw std::runtime_error("setLatticeSize must be called before initialize");
        if (rng != BFM_RNG_INTHASH && rng != BFM_RNG_SARU && rng != BFM_RNG_PHILOX)
            throw std::runtime_error("random number generator " + std::to_string(rng) +
                                     " is not provided by this build (IntHash = 1, Saru = 2, Philox = 3)");
        /* initializeBondTable (.cu:1516-1559): exactly 108 allowed bonds */
        unsigned nAllowed = 0;
        for (int i = 0; i < 512; ++i) nAllowed += forbidden[i] ? 0 : 1;
        if (nAllowed != 108)
            throw std::runtime_error("Wrong bond-set! Expected 108 allowed bonds, but got " + std::to_string(nAllowed));
        std::memset(&bonds, 0, sizeof(bonds));
        for (uint32_t dz = 0; dz < 8; ++dz)
            for (uint32_t dy = 0; dy < 8; ++dy)
                for (uint32_t dx = 0; dx < 8; ++dx)
                    if (forbidden[dx | (dy << 3) | (dz << 6)]) {
                        const uint32_t code = zcode(dx, dy, dz);
                        bonds.forbidden[code >> 5] |= 1u << (code & 31);
                    }

        Lm = (uint32_t)std::max(L[0], std::max(L[1], L[2]));
        keyBits = 3 * ilog2(Lm);
        latWords = ((size_t)Lm * Lm * Lm) / 32;
        g.open = 0;
        for (int a = 0; a < 3; ++a) {
            g.m[a] = dilate3((uint32_t)L[a] - 1) << a;
            g.top[a] = periodic[a] ? 0u : dilate3((uint32_t)L[a] - 2) << a;
            if (!periodic[a]) g.open |= 1u << a;
        }
        /* along a non-periodic axis every cube lies inside the box: corner in 0 .. L-2 */
        for (uint32_t i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a)
                if (!periodic[a] && (xyz[3 * (size_t)i + a] < 0 || xyz[3 * (size_t)i + a] > (int64_t)L[a] - 2))
                    throw InvalidArgument("monomer " + std::to_string(i) + " lies outside the box along the non-periodic axis " +
                                          std::string(1, "xyz"[a]));

        /* graph colouring (initializeSpeciesSorting, .cu:1561-1686) */
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = 0; j < deg[i]; ++j)
                if (nbr[(size_t)i * 8 + j] >= n)
                    throw InvalidArgument("bond partner id out of range for monomer " + std::to_string(i));
        colorOnDevice = 0;
        if (coloringMode == 1) {
            CK(cudaSetDevice(gpu));
            colorOnDevice = color_graph_device(n, deg.data(), nbr.data(), true, color);
        }
        if (!colorOnDevice) color = color_graph(n, deg.data(), nbr.data(), true);
        nSpecies = 0;
        for (uint32_t i = 0; i < n; ++i) nSpecies = std::max(nSpecies, color[i] + 1);
        std::vector<uint32_t> count(nSpecies, 0);
        for (uint32_t i = 0; i < n; ++i) ++count[color[i]];
        spec.assign(nSpecies, Species{0, 0});
        uint32_t off = 0;
        nmax = 0;
        for (uint32_t c = 0; c < nSpecies; ++c) {
            spec[c].off = off;
            spec[c].n = count[c];
            nmax = std::max(nmax, count[c]);
            off += (count[c] + kSlabAlign - 1) / kSlabAlign * kSlabAlign;
        }
        npad = std::max(off, kSlabAlign);
        maxdeg = 0;
        for (uint32_t i = 0; i < n; ++i) maxdeg = std::max<uint32_t>(maxdeg, deg[i]);

        /* slot order inside a species: ascending original id (.cu:1648-1650) */
        std::vector<uint32_t> o2s(n), s2o(npad, kNoId);
        {
            std::vector<uint32_t> next(nSpecies);
            for (uint32_t c = 0; c < nSpecies; ++c) next[c] = spec[c].off;
            for (uint32_t i = 0; i < n; ++i) {
                o2s[i] = next[color[i]]++;
                s2o[o2s[i]] = i;
            }
        }

        /* wrapped codes + image counters (initializeSortedMonomerPositions, .cu:2066-2139),
         * occupation lattice (initializeLattices, .cu:2141-2236) and the
         * excluded-volume / bond checks of checkSystem (.cu:2789-2900) */
        std::vector<uint32_t> hpos(npad, 0);
        std::vector<int32_t> himg(3 * (size_t)npad, 0);
        std::vector<uint32_t> hlat(latWords, 0);
        std::vector<uint64_t> cells(((size_t)Lm * Lm * Lm + 63) / 64, 0);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t slot = o2s[i];
            uint32_t w[3];
            for (int a = 0; a < 3; ++a) {
                const int64_t v = xyz[3 * (size_t)i + a];
                const int64_t La = (int64_t)L[a];
                int64_t q = v / La;
                int64_t r = v - q * La;
                if (r < 0) { r += La; --q; }
                w[a] = (uint32_t)r;
                himg[(size_t)a * npad + slot] = (int32_t)q;
            }
            const uint32_t code = zcode(w[0], w[1], w[2]);
            hpos[slot] = code;
            if ((hlat[code >> 5] >> (code & 31)) & 1u)
                throw InvalidArgument("two monomers share the lattice position of monomer " + std::to_string(i));
            hlat[code >> 5] |= 1u << (code & 31);
            for (int c = 0; c < 8; ++c) {
                const uint32_t cc = zcode((w[0] + (c & 1)) & (uint32_t)(L[0] - 1), (w[1] + ((c >> 1) & 1)) & (uint32_t)(L[1] - 1),
                                          (w[2] + ((c >> 2) & 1)) & (uint32_t)(L[2] - 1));
                if ((cells[cc >> 6] >> (cc & 63)) & 1u)
                    throw InvalidArgument("excluded volume violated: the 2x2x2 cube of monomer " + std::to_string(i) + " overlaps another one");
                cells[cc >> 6] |= 1ull << (cc & 63);
            }
        }
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = 0; j < deg[i]; ++j) {
                const uint32_t k = nbr[(size_t)i * 8 + j];
                const int64_t dx = (int64_t)xyz[3 * (size_t)k] - xyz[3 * (size_t)i];
                const int64_t dy = (int64_t)xyz[3 * (size_t)k + 1] - xyz[3 * (size_t)i + 1];
                const int64_t dz = (int64_t)xyz[3 * (size_t)k + 2] - xyz[3 * (size_t)i + 2];
                if (dx < -3 || dx > 3 || dy < -3 || dy > 3 || dz < -3 || dz > 3 ||
                    forbidden[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)])
                    throw InvalidArgument("bond " + std::to_string(i) + "-" + std::to_string(k) + " (" + std::to_string(dx) + "," +
                                          std::to_string(dy) + "," + std::to_string(dz) + ") is not in the bond set");
            }
        std::vector<uint32_t> hnbr((size_t)std::max(maxdeg, 1u) * npad, 0);
        std::vector<uint8_t> hdeg(npad, 0);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t slot = o2s[i];
            hdeg[slot] = deg[i];
            for (uint32_t j = 0; j < deg[i]; ++j) hnbr[(size_t)j * npad + slot] = o2s[nbr[(size_t)i * 8 + j]];
        }
        /* reverse rows: the m-th bond of i to k pairs with the m-th bond of k to i */
        std::vector<uint8_t> hrev((size_t)std::max(maxdeg, 1u) * npad, 0);
        storedBonds = true;
        for (uint32_t i = 0; i < n && storedBonds; ++i)
            for (uint32_t j = 0; j < deg[i]; ++j) {
                const uint32_t k = nbr[(size_t)i * 8 + j];
                uint32_t occ = 0;
                for (uint32_t t = 0; t < j; ++t) occ += nbr[(size_t)i * 8 + t] == k;
                int r = -1;
                for (uint32_t t = 0, seen = 0; t < deg[k]; ++t)
                    if (nbr[(size_t)k * 8 + t] == i && seen++ == occ) {
                        r = (int)t;
                        break;
                    }
                if (r < 0 || k == i) {
                    storedBonds = false;
                    break;
                }
                hrev[(size_t)j * npad + o2s[i]] = (uint8_t)r;
            }

        CK(cudaSetDevice(gpu));
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        const size_t nbrRows = std::max(maxdeg, 1u);
        dalloc(d_pos, npad); dalloc(d_pos2, npad);
        dalloc(d_img, 3 * (size_t)npad); dalloc(d_img2, 3 * (size_t)npad);
        dalloc(d_nbr, nbrRows * npad); dalloc(d_nbr2, nbrRows * npad);
        dalloc(d_deg, npad); dalloc(d_deg2, npad);
        dalloc(d_rev, nbrRows * npad); dalloc(d_rev2, nbrRows * npad);
        dalloc(d_bcode, std::max<size_t>(nbrRows, 2) * npad); /* rows 0 and 1 interleaved: bc_index */
        dalloc(d_s2o, npad); dalloc(d_s2o2, npad); dalloc(d_o2s, n);
        dalloc(d_flags, npad);
        dalloc(d_lat, latWords);
        dalloc(d_tmp, 2 * latWords);
        dalloc(d_spec, nSpecies);
        dalloc(d_counters, 4);
        dalloc(d_perm, npad); dalloc(d_inv, npad); dalloc(d_iota, npad); dalloc(d_keys, npad);
        dalloc(d_out, 3 * (size_t)n);
        for (int b = 0; b < 2; ++b) {
            dalloc(d_sched[b], std::max(kChunk, 256u * 2u));
            CK(cudaMallocHost((void **)&h_sched[b], std::max(kChunk, 256u * 2u) * sizeof(Substep)));
            CK(cudaEventCreateWithFlags(&schedFree[b], cudaEventDisableTiming));
        }
        CK(cudaMallocHost((void **)&h_out, 3 * (size_t)n * sizeof(int32_t)));
        CK(cudaMallocHost((void **)&h_flag, sizeof(unsigned int)));
        *h_flag = 0;
        {
            cub::DeviceRadixSort::SortPairs(nullptr, cubBytes, d_pos, d_keys, d_iota, d_perm, (int)nmax, 0, (int)keyBits, stream);
            CK(cudaMalloc(&d_cub, std::max<size_t>(cubBytes, 16)));
        }
        std::vector<uint32_t> iota(npad);
        for (uint32_t i = 0; i < npad; ++i) iota[i] = i;
        CK(cudaMemcpyAsync(d_pos, hpos.data(), npad * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_img, himg.data(), himg.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_nbr, hnbr.data(), hnbr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_deg, hdeg.data(), npad, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_rev, hrev.data(), hrev.size(), cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(d_bcode, 0, std::max<size_t>(nbrRows, 2) * npad * sizeof(uint16_t), stream));
        CK(cudaMemcpyAsync(d_s2o, s2o.data(), npad * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_o2s, o2s.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_lat, hlat.data(), latWords * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_spec, spec.data(), nSpecies * sizeof(Species), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_iota, iota.data(), npad * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_perm, iota.data(), npad * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(d_tmp, 0, 2 * latWords * sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(d_flags, 0, npad, stream));
        CK(cudaMemsetAsync(d_counters, 0, 4 * sizeof(unsigned long long), stream));
        dalloc(d_bar, 1);
        CK(cudaMemsetAsync(d_bar, 0, sizeof(GridBarrier), stream));
        configureSweep();
        CK(cudaStreamSynchronize(stream));
        substepCounter = 0;
        nAttempts = 0;
        initialized = true;
        sortedFresh = false;
        /* the reference sorts at initialize when age != 0 (.cu:2511-2512) and
         * at the first step when age % stepsBetweenSortings == 0 (.cu:3005);
         * the Z-order sort is idempotent, so sorting here always gives the
         * same slot order before the first substep. */
        spatialSort();
        hostPosValid = false;
    }

    /* recompute the stored bond codes from the positions (after set-up, a
     * re-sort, or a run of the per-substep kernels, which do not keep them) */
    void refreshBondCodes()
    {
        if (maxdeg == 0) return;
        const int blocks = (int)std::min<uint32_t>((npad + kThreads - 1) / kThreads, 148 * 16);
        k_bondcodes<<<blocks, kThreads, 0, stream>>>(d_pos, d_nbr, d_deg, d_bcode, npad);
        CK(cudaGetLastError());
    }

    /* Persistent-kernel launch shape: as many CTAs as can be co-resident (a
     * cooperative launch needs them all resident); each CTA's candidate
     * list holds its worst case (every monomer it checks is a candidate),
     * in shared memory when that fits. */
    int sweepMode = 0;
    uint32_t sweepWindow = 0;
    int forcedShape = -1; /* -1 automatic; 0..2 bond mode; +3: candidate lists in global memory; 6 windowed */
    int extraRounds = 0;  /* windowed shapes: rounds of items per thread beyond the fewest (smaller CTAs) */

    /* launch-shape autotuner: on the first chunk of the next run, each
     * candidate shape runs a trial launch of an equal share of the chunk's
     * substeps (part of the run: every shape gives the same trajectory),
     * timed with events; the fastest per attempted move is kept unless the
     * automatic shape is within 3% of it */
    struct ShapeTrial {
        int shape, extra, threads;
        double nsPerMove;
    };
    bool autotune = false, tuned = false;
    std::vector<ShapeTrial> trials;
    int sweepThreads = kSweepThreads;
    uint32_t sweepTotal = 0; /* windowed kernel: most items of all colours one CTA owns */
    bool sweepGlobalList = false; /* k_sweep: candidate lists in global memory */

    /* Persistent-kernel launch shape: one CTA per SM (cooperative launch,
     * all CTAs resident); each CTA owns 1/grid of every colour slab.  The
     * candidate list holds the CTA's worst case (every monomer a candidate).
     * Staged mode when the CTA's segments and list fit in shared memory. */
    template <int RNG, int MODE>
    bool configureFor(int smCount, size_t smemLimit)
    {
        int blocks = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_sweep<RNG, MODE>, kSweepThreads, 0));
        if (blocks < 1) throw std::runtime_error("persistent sweep kernel does not fit on an SM");
        const uint32_t grid = (uint32_t)smCount; /* one CTA per SM */
        const uint32_t per = (nmax + grid - 1) / grid + 1u;
        const uint32_t cap = std::max<uint32_t>(32u, per);
        const uint32_t W = ((per + 15u) & ~15u) + 32u;
        size_t smem = kWinTableBytes;
        bool globalList = forcedShape >= 3;
        if (MODE == SWEEP_STAGED) {
            if (globalList) return false;
            smem = StageLayout{W}.bytes(cap);
            if (smem > smemLimit) return false;
        } else {
            if ((size_t)cap * sizeof(uint2) > kSweepSmemListMax) globalList = true;
            if (!globalList) smem += (size_t)cap * sizeof(uint2);
            if (MODE == SWEEP_STORED) {
                smem += kBondFirstBytes;
                if (smem > smemLimit) return false;
            }
        }
        raise_smem_limit((const void *)k_sweep<RNG, MODE>, smem);
        int fit = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_sweep<RNG, MODE>, kSweepThreads, smem));
        if (fit < 1) return false;
        sweepGrid = (int)grid;
        sweepCap = cap;
        sweepSmem = smem;
        sweepGlobalList = globalList;
        sweepWindow = W;
        sweepMode = MODE;
        sweepThreads = kSweepThreads;
        return true;
    }

    /* the windowed kernel (shape 6 + variant): one CTA per SM (variants
     * 0..2) or one cluster of 8 or 16 CTAs (3, 4); positions, directions and
     * both candidate lists in shared memory */
    template <int RNG>
    bool configureWindowed(int smCount, size_t smemLimit, int variant)
    {
        if (nSpecies > kWinMaxSpecies) return false;
        const uint32_t cluster = (uint32_t)kWinCluster[variant];
        const uint32_t grid = cluster ? cluster : (uint32_t)smCount;
        const uint32_t per = (nmax + grid - 1) / grid + 1u;
        const uint32_t W = (per + 15u) & ~15u;
        /* fewest rounds of U items per thread at <= 1024 threads (plus
         * `extraRounds`, which the autotuner may add for smaller CTAs), then
         * the fewest warps for that many rounds (at least 2: warp 0 watches
         * the barriers) */
        const uint32_t U = (uint32_t)kWinU[variant];
        const uint32_t rounds = (per + U * 1024u - 1u) / (U * 1024u) + (uint32_t)extraRounds;
        const uint32_t threads = std::max<uint32_t>(64u, 32u * ((per + 32u * U * rounds - 1u) / (32u * U * rounds)));
        uint32_t P = 0; /* most items of all colours one CTA owns */
        for (uint32_t c = 0; c < nSpecies; ++c) P += (spec[c].n + grid - 1) / grid;
        P = (P + 15u) & ~15u;
        const size_t smem = WinLayout{W, threads, P, kWinBondFirst[variant]}.bytes();
        if (smem > smemLimit) return false;
        const void *fn = win_kernel<RNG>(variant);
        raise_smem_limit(fn, smem);
        int fit = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, (int)threads, smem));
        if (fit < 1) return false;
        if (cluster) {
            if (cluster > 8) CK(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cluster);
            cfg.blockDim = dim3(threads);
            cfg.dynamicSmemBytes = smem;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = cluster;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess) {
                (void)cudaGetLastError();
                return false;
            }
            if (clusters < 1) return false;
        }
        sweepGrid = (int)grid;
        sweepCap = W;
        sweepSmem = smem;
        sweepWindow = W;
        sweepMode = SWEEP_WINDOWED + variant;
        sweepGlobalList = false;
        sweepThreads = (int)threads;
        sweepTotal = P;
        return true;
    }

    template <int RNG>
    void configureRng(int smCount, size_t smemLimit)
    {
        if (forcedShape >= SWEEP_WINDOWED) {
            if (!storedBonds || !configureWindowed<RNG>(smCount, smemLimit, forcedShape - SWEEP_WINDOWED))
                throw std::runtime_error("the requested persistent-kernel shape is not available for this system");
            return;
        }
        if (forcedShape >= 0) {
            const int m = forcedShape % 3;
            bool ok = false;
            if (m == SWEEP_STAGED && storedBonds) ok = configureFor<RNG, SWEEP_STAGED>(smCount, smemLimit);
            else if (m == SWEEP_STORED && storedBonds) ok = configureFor<RNG, SWEEP_STORED>(smCount, smemLimit);
            else if (m == SWEEP_GATHER) ok = configureFor<RNG, SWEEP_GATHER>(smCount, smemLimit);
            if (!ok) throw std::runtime_error("the requested persistent-kernel shape is not available for this system");
            return;
        }
        if (storedBonds) {
            if (nmax / (uint32_t)smCount >= kWinBondFirstItems && configureWindowed<RNG>(smCount, smemLimit, 2)) return;
            if (configureWindowed<RNG>(smCount, smemLimit, 1)) return; /* 2 items in flight per thread */
            if (configureFor<RNG, SWEEP_STAGED>(smCount, smemLimit)) return;
            if (configureFor<RNG, SWEEP_STORED>(smCount, smemLimit)) return;
        }
        if (!configureFor<RNG, SWEEP_GATHER>(smCount, smemLimit))
            throw std::runtime_error("persistent sweep kernel does not fit on an SM");
    }

    void configureSweep()
    {
        int dev = 0, sms = 0, optin = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        if (npad >= (1u << 28)) throw std::runtime_error("more than 2^28 monomer slots are not supported");
        const size_t limit = (size_t)optin > 16384 ? (size_t)optin - 16384 : (size_t)optin; /* room for the static tables */
        if (rng == BFM_RNG_SARU)
            configureRng<RNG_SARU>(sms, limit);
        else if (rng == BFM_RNG_PHILOX)
            configureRng<RNG_PHILOX>(sms, limit);
        else
            configureRng<RNG_INTHASH>(sms, limit);
        dfree(d_glist);
        if (sweepGlobalList) dalloc(d_glist, (size_t)sweepGrid * sweepCap);
    }

    void launchSweep(const Substep *sched, uint32_t k0, uint32_t k1)
    {
        Sys s = sys();
        uint2 *gl = sweepGlobalList ? d_glist : nullptr;
        uint32_t cap = sweepCap;
        GridBarrier *bar = d_bar;
        unsigned long long to = timeoutNs;
        uint32_t md = maxdeg;
        uint32_t win = sweepWindow;
        void *args[] = {&s, (void *)&sched, &k0, &k1, &bar, &gl, &cap, &to, &md, &win};
        CK(cudaMemsetAsync(d_bar, 0, sizeof(GridBarrier), stream)); /* the counting barrier starts at 0 */
        if (sweepMode >= SWEEP_WINDOWED) {
            uint32_t ns = nSpecies, pt = sweepTotal;
            void *wargs[] = {&s, (void *)&sched, &k0, &k1, &bar, &to, &md, &win, &ns, &pt};
            const int v = sweepMode - SWEEP_WINDOWED;
            const void *wf = rng == BFM_RNG_SARU     ? win_kernel<RNG_SARU>(v)
                             : rng == BFM_RNG_PHILOX ? win_kernel<RNG_PHILOX>(v)
                                                     : win_kernel<RNG_INTHASH>(v);
            if (kWinCluster[v]) { /* one cluster: hardware cluster barriers */
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)sweepGrid);
                cfg.blockDim = dim3((unsigned)sweepThreads);
                cfg.dynamicSmemBytes = sweepSmem;
                cfg.stream = stream;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = (unsigned)sweepGrid;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                CK(cudaLaunchKernelExC(&cfg, wf, wargs));
                return;
            }
            CK(cudaLaunchCooperativeKernel(wf, dim3(sweepGrid), dim3(sweepThreads), wargs, sweepSmem, stream));
            return;
        }
        const void *fn = nullptr;
        if (rng == BFM_RNG_SARU)
            fn = sweepMode == SWEEP_STAGED ? (const void *)k_sweep<RNG_SARU, SWEEP_STAGED>
                 : sweepMode == SWEEP_STORED ? (const void *)k_sweep<RNG_SARU, SWEEP_STORED>
                                             : (const void *)k_sweep<RNG_SARU, SWEEP_GATHER>;
        else if (rng == BFM_RNG_PHILOX)
            fn = sweepMode == SWEEP_STAGED ? (const void *)k_sweep<RNG_PHILOX, SWEEP_STAGED>
                 : sweepMode == SWEEP_STORED ? (const void *)k_sweep<RNG_PHILOX, SWEEP_STORED>
                                             : (const void *)k_sweep<RNG_PHILOX, SWEEP_GATHER>;
        else
            fn = sweepMode == SWEEP_STAGED ? (const void *)k_sweep<RNG_INTHASH, SWEEP_STAGED>
                 : sweepMode == SWEEP_STORED ? (const void *)k_sweep<RNG_INTHASH, SWEEP_STORED>
                                             : (const void *)k_sweep<RNG_INTHASH, SWEEP_GATHER>;
        CK(cudaLaunchCooperativeKernel(fn, dim3(sweepGrid), dim3(kSweepThreads), args, sweepSmem, stream));
    }

    /* doSpatialSorting (.cu:1835-1943): per species, order slots by the
     * Z-order code of the wrapped position (the position code itself). */
    void spatialSort()
    {
        for (uint32_t c = 0; c < nSpecies; ++c) {
            if (spec[c].n == 0) continue;
            size_t bytes = cubBytes;
            CK(cub::DeviceRadixSort::SortPairs(d_cub, bytes, d_pos + spec[c].off, d_keys, d_iota + spec[c].off,
                                               d_perm + spec[c].off, (int)spec[c].n, 0, (int)keyBits, stream));
        }
        const int blocks = (int)std::min<uint32_t>((npad + kThreads - 1) / kThreads, 148 * 16);
        k_invert<<<blocks, kThreads, 0, stream>>>(d_perm, d_inv, npad);
        k_permute<<<blocks, kThreads, 0, stream>>>(d_perm, d_inv, npad, maxdeg, d_pos, d_img, d_nbr, d_deg, d_s2o, d_rev,
                                                   d_pos2, d_img2, d_nbr2, d_deg2, d_s2o2, d_rev2, d_o2s);
        CK(cudaGetLastError());
        std::swap(d_pos, d_pos2);
        std::swap(d_img, d_img2);
        std::swap(d_nbr, d_nbr2);
        std::swap(d_deg, d_deg2);
        std::swap(d_rev, d_rev2);
        refreshBondCodes();
        std::swap(d_s2o, d_s2o2);
        /* the captured graphs hold the old pointers */
        for (auto &ge : graph)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
        graphRng = -1;
        sortedFresh = true;
    }

    int checkBlocks() const
    {
        const uint32_t want = std::max<uint32_t>((nmax + kThreads - 1) / kThreads, (uint32_t)((latWords / 4 + kThreads - 1) / kThreads));
        return (int)std::max<uint32_t>(1, std::min<uint32_t>(want, 148u * 64u));
    }
    int performBlocks() const { return (int)std::max<uint32_t>(1, std::min<uint32_t>((nmax + kThreads - 1) / kThreads, 148u * 64u)); }

    /* event pairs around every sweep-kernel launch when profiling */
    bool profiling = false;
    std::vector<cudaEvent_t> profEvents;
    size_t profUsed = 0;
    void profMark()
    {
        if (!profiling) return;
        if (profUsed == profEvents.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            profEvents.push_back(e);
        }
        CK(cudaEventRecord(profEvents[profUsed++], stream));
    }

    void launchSubstep(const Substep *sched, uint32_t k)
    {
        const Sys s = sys();
        profMark();
        if (rng == BFM_RNG_SARU)
            k_check<RNG_SARU><<<checkBlocks(), kThreads, 0, stream>>>(s, sched, k);
        else if (rng == BFM_RNG_PHILOX)
            k_check<RNG_PHILOX><<<checkBlocks(), kThreads, 0, stream>>>(s, sched, k);
        else
            k_check<RNG_INTHASH><<<checkBlocks(), kThreads, 0, stream>>>(s, sched, k);
        profMark();
        profMark();
        k_perform<<<performBlocks(), kThreads, 0, stream>>>(s, sched, k);
        profMark();
    }

    /* run nMCS in the current launch path (graphs replaced by direct
     * launches) with CUDA events around every sweep-kernel launch on the
     * handle's stream: summed device time, launches, attempted moves */
    void timeKernels(uint32_t nMCS, double *ms, uint64_t *launches, uint64_t *attempts)
    {
        const int saved = launchMode;
        if (launchMode == 1) launchMode = 2;
        profiling = true;
        profUsed = 0;
        const uint64_t a0 = nAttempts;
        try {
            run(nMCS);
        } catch (...) {
            profiling = false;
            launchMode = saved;
            throw;
        }
        profiling = false;
        launchMode = saved;
        double t = 0;
        for (size_t i = 0; i + 1 < profUsed; i += 2) {
            float a = 0;
            CK(cudaEventElapsedTime(&a, profEvents[i], profEvents[i + 1]));
            t += a;
        }
        *ms = t;
        *launches = profUsed / 2;
        *attempts = nAttempts - a0;
    }

    /* substeps per captured graph: a whole number of MCS */
    uint32_t graphSubsteps() const { return std::max(1u, kGraphSubsteps / nSpecies) * nSpecies; }

    void buildGraph(int b)
    {
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (uint32_t k = 0; k < graphSubsteps(); ++k) launchSubstep(d_sched[b], k);
        CK(cudaStreamEndCapture(stream, &gr));
        CK(cudaGraphInstantiate(&graph[b], gr, 0));
        CK(cudaGraphDestroy(gr));
    }

    /* the autotuner's trials on substeps [0, m) of the uploaded chunk, then
     * the rest of the chunk with the chosen shape; returns the launches.  A
     * first piece with the automatic shape warms the caches (untimed); then
     * every candidate runs two timed pieces, in two rounds, and keeps the
     * faster -- so neither the cold start nor a drift of the acceptance
     * rate along the chunk favours one shape. */
    uint64_t tuneShapes(const Substep *sched, const Substep *hs, uint32_t m)
    {
        const int savedShape = forcedShape, savedExtra = extraRounds;
        /* candidates: automatic first, then every other shape that fits */
        std::vector<std::pair<int, int>> cand = {{-1, 0}};
        const int autoMode = sweepMode;
        for (int sh : {6, 7, 8, 9, 10, 1, 2})
            if (sh != autoMode) cand.push_back({sh, 0});
        cand.push_back({autoMode >= SWEEP_WINDOWED ? autoMode : 7, 1});
        std::vector<std::pair<int, int>> ok;
        for (auto &c : cand) {
            forcedShape = c.first;
            extraRounds = c.second;
            try {
                configureSweep();
            } catch (std::runtime_error const &) {
                continue; /* this shape does not fit the system */
            }
            ok.push_back(c);
        }
        const uint32_t pieces = 2u * (uint32_t)ok.size() + 1u;
        const uint32_t piece = std::max<uint32_t>(1, m / pieces / nSpecies) * nSpecies;
        uint32_t k = 0;
        uint64_t launches = 0;
        trials.clear();
        std::vector<cudaEvent_t> ev;
        std::vector<uint64_t> att;
        std::vector<size_t> who;
        auto use = [&](const std::pair<int, int> &c) {
            forcedShape = c.first;
            extraRounds = c.second;
            configureSweep();
        };
        if (!ok.empty() && k + piece <= m) { /* warm-up piece, untimed */
            use(ok[0]);
            launchSweep(sched, k, k + piece);
            ++launches;
            k += piece;
        }
        for (int round = 0; round < 2; ++round)
            for (size_t ci = 0; ci < ok.size(); ++ci) {
                if (k + piece > m) break;
                use(ok[ci]);
                if (round == 0) trials.push_back({ok[ci].first < 0 ? sweepMode : ok[ci].first, ok[ci].second, sweepThreads, 0.0});
                cudaEvent_t e0, e1;
                CK(cudaEventCreate(&e0));
                CK(cudaEventCreate(&e1));
                ev.push_back(e0);
                ev.push_back(e1);
                CK(cudaEventRecord(e0, stream));
                launchSweep(sched, k, k + piece);
                CK(cudaEventRecord(e1, stream));
                ++launches;
                uint64_t a = 0;
                for (uint32_t j = k; j < k + piece; ++j) a += spec[hs[j].species].n;
                att.push_back(a);
                who.push_back(ci);
                k += piece;
            }
        CK(cudaStreamSynchronize(stream));
        for (size_t t = 0; t < who.size(); ++t) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[2 * t], ev[2 * t + 1]));
            const double ns = ms * 1e6 / std::max<double>((double)att[t], 1.0);
            double &best = trials[who[t]].nsPerMove;
            if (best == 0.0 || ns < best) best = ns;
        }
        for (auto e : ev) cudaEventDestroy(e);
        size_t best = 0;
        for (size_t i = 0; i < trials.size(); ++i)
            if (trials[i].nsPerMove > 0.0 && trials[i].nsPerMove < trials[best].nsPerMove) best = i;
        /* keep the automatic shape unless another is more than 3% faster */
        if (!trials.empty() && trials[best].nsPerMove < 0.97 * trials[0].nsPerMove) {
            forcedShape = trials[best].shape;
            extraRounds = trials[best].extra;
        } else {
            forcedShape = savedShape;
            extraRounds = savedExtra;
        }
        configureSweep();
        tuned = true;
        if (k < m) {
            launchSweep(sched, k, m);
            ++launches;
        }
        return launches;
    }

    /* runSimulationOnGPU (.cu:2902-3400) */
    void run(uint32_t nMCS)
    {
        if (!initialized) throw std::runtime_error("initialize must be called before runSimulationOnGPU");
        hostPosValid = false;
        if (graphRng != rng) {
            for (auto &ge : graph)
                if (ge) {
                    cudaGraphExecDestroy(ge);
                    ge = nullptr;
                }
            graphRng = rng;
        }
        /* the filter analysis runs the per-substep kernels, which count */
        const int mode = filterStats ? 2 : launchMode;
        if (filterStats) {
            if (!d_fstats) dalloc(d_fstats, (size_t)kChunk * kFilters);
            resetFilterStats();
        }
        R250 &r250 = global_r250();
        std::lock_guard<std::mutex> lock(g_r250_mutex);
        CK(cudaEventRecord(ev0, stream));
        uint64_t launches = 0;
        uint32_t iStep = 0;
        int b = 0;
        const uint32_t cap = mode == 1 ? graphSubsteps() : (kChunk / nSpecies) * nSpecies;
        while (iStep < nMCS) {
            /* one schedule chunk: whole MCS only, ending before a re-sort */
            CK(cudaEventSynchronize(schedFree[b]));
            Substep *hs = h_sched[b];
            uint32_t m = 0;
            bool sortFirst = false;
            const uint32_t step0 = iStep;
            while (iStep < nMCS && m + nSpecies <= cap) {
                const int64_t a = age + iStep; /* mAge, advanced once per MCS (.cu:3002) */
                if (a % sortEvery == 0) {      /* .cu:3005 */
                    if (iStep != step0) break;
                    sortFirst = true;
                }
                for (uint32_t sub = 0; sub < nSpecies; ++sub) {
                    Substep &d = hs[m++];
                    const uint64_t currentAge = (uint64_t)a + (uint64_t)iStep * nSpecies + sub; /* .cu:3049 */
                    d.species = (uint16_t)((uint64_t)r250.next() % nSpecies);                /* .cu:3065 */
                    d.seed = r250.next();                                                    /* .cu:3066 */
                    d.iter = (uint32_t)currentAge;
                    d.iterHi = (uint32_t)(currentAge >> 32);
                    d.buf = (uint16_t)(substepCounter++ & 1u);
                    nAttempts += spec[d.species].n;
                }
                ++iStep;
            }
            if (sortFirst && !sortedFresh) spatialSort();
            CK(cudaMemcpyAsync(d_sched[b], hs, m * sizeof(Substep), cudaMemcpyHostToDevice, stream));
            CK(cudaEventRecord(schedFree[b], stream));
            if (filterStats) CK(cudaMemsetAsync(d_fstats, 0, (size_t)m * kFilters * sizeof(unsigned long long), stream));
            if (mode == 0 && autotune && !tuned && m >= 2 * nSpecies) {
                launches += tuneShapes(d_sched[b], hs, m);
            } else if (mode == 0) {
                profMark();
                launchSweep(d_sched[b], 0, m);
                profMark();
                launches += 1;
            } else if (mode == 1 && m == cap) {
                if (!graph[b]) buildGraph(b);
                CK(cudaGraphLaunch(graph[b], stream));
                launches += 2 * (uint64_t)m;
            } else {
                for (uint32_t k = 0; k < m; ++k) launchSubstep(d_sched[b], k);
                launches += 2 * (uint64_t)m;
            }
            CK(cudaGetLastError());
            if (filterStats) accumulateFilterStats(hs, m);
            sortedFresh = false;
            b ^= 1;
        }
        age += nMCS;
        /* the split kernels leave the target buffer of their last substep
         * set; the persistent kernel clears its own before it returns */
        if (mode != 0) {
            CK(cudaMemsetAsync(d_tmp, 0, 2 * latWords * sizeof(uint32_t), stream));
            refreshBondCodes();
        }
        CK(cudaEventRecord(ev1, stream));
        if (mode == 0) CK(cudaMemcpyAsync(h_flag, &d_bar->err, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
        CK(cudaEventSynchronize(ev1));
        CK(cudaStreamSynchronize(stream));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        lastRunMs = ms;
        lastLaunches = launches;
        CK(cudaGetLastError());
        if (mode == 0 && *h_flag) {
            CK(cudaMemsetAsync(d_bar, 0, sizeof(GridBarrier), stream));
            CK(cudaStreamSynchronize(stream));
            throw DeviceTimeout("a grid barrier of the persistent sweep kernel timed out; the positions of this run are not valid");
        }
    }

    /* ------------------------------------------ filter statistics */
    unsigned long long *d_fstats = nullptr;
    std::vector<double> fsum, fsum2, fmin, fmax, fcnt; /* [species][filter], per run as .cu:2926-2936 */

    void resetFilterStats()
    {
        const size_t z = (size_t)nSpecies * kFilters;
        fsum.assign(z, 0.0);
        fsum2.assign(z, 0.0);
        fmin.assign(z, (double)n);
        fmax.assign(z, 0.0);
        fcnt.assign(z, 0.0);
    }

    /* counts of one chunk of m substeps into the per-species statistics (.cu:3316-3330) */
    void accumulateFilterStats(const Substep *hs, uint32_t m)
    {
        std::vector<unsigned long long> c((size_t)m * kFilters);
        CK(cudaMemcpyAsync(c.data(), d_fstats, c.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (uint32_t k = 0; k < m; ++k)
            for (int f = 0; f < kFilters; ++f) {
                const size_t at = (size_t)hs[k].species * kFilters + f;
                const double x = (double)c[(size_t)k * kFilters + f];
                fsum[at] += x;
                fsum2[at] += x * x;
                fmin[at] = std::min(fmin[at], x);
                fmax[at] = std::max(fmax[at], x);
                fcnt[at] += 1.0;
            }
    }

    /* ------------------------------------------------ chain analysis */
    LinearChains chains;
    bool chainsReady = false, haveOrigin = false;
    uint32_t *d_coff = nullptr, *d_cmem = nullptr, *d_cfirst = nullptr, *d_cmid = nullptr, *d_clast = nullptr;
    ChainSums *d_csum = nullptr;
    ChainOrigin *d_corg = nullptr;
    double *d_cbox = nullptr, *d_cre2 = nullptr, *d_crg2 = nullptr, *d_ccom = nullptr, *d_cout = nullptr;

    void releaseAnalyzer()
    {
        dfree(d_coff); dfree(d_cmem); dfree(d_cfirst); dfree(d_cmid); dfree(d_clast); dfree(d_csum); dfree(d_corg);
        dfree(d_cbox); dfree(d_cre2); dfree(d_crg2); dfree(d_ccom); dfree(d_cout);
        chainsReady = haveOrigin = false;
    }

    uint32_t nChains() const { return (uint32_t)chains.first.size(); }

    /* linear chains of the system by the reference analyzer's rule */
    void analyzerInit()
    {
        if (!initialized) throw std::runtime_error("initialize must be called first");
        LinearChains lc = linear_chains(n, deg.data(), nbr.data());
        releaseAnalyzer();
        chains = std::move(lc);
        const uint32_t nc = nChains();
        dalloc(d_coff, nc + 1); dalloc(d_cmem, (size_t)n); dalloc(d_cfirst, nc); dalloc(d_cmid, nc); dalloc(d_clast, nc);
        dalloc(d_csum, nc); dalloc(d_corg, nc); dalloc(d_cbox, 3); dalloc(d_cre2, nc); dalloc(d_crg2, nc);
        dalloc(d_ccom, 3 * (size_t)nc); dalloc(d_cout, 16);
        CK(cudaMemcpyAsync(d_coff, chains.off.data(), (nc + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_cmem, chains.members.data(), (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_cfirst, chains.first.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_cmid, chains.middle.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_clast, chains.last.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
        chainsReady = true;
        haveOrigin = false;
    }

    /* observables of the current state (out: 11 doubles); setOrigin makes
     * the current state the time origin of the mean-square displacements */
    void analyze(double *out, bool setOrigin)
    {
        if (!chainsReady) throw std::runtime_error("bfm_analyzer_init must be called first");
        const uint32_t nc = nChains();
        const int blocks = (int)std::min<uint32_t>((npad + kThreads - 1) / kThreads, 148 * 16);
        k_unpack<<<blocks, kThreads, 0, stream>>>(d_pos, d_img, d_s2o, npad, (int32_t)L[0], (int32_t)L[1], (int32_t)L[2], d_out);
        const int cblocks = (int)std::min<uint32_t>((nc + 7) / 8, 148 * 8);
        k_chain_sums<<<std::max(cblocks, 1), 256, 0, stream>>>(d_out, d_coff, d_cmem, nc, d_csum);
        k_chain_observables<<<1, kAnalyzeThreads, 0, stream>>>(d_out, d_csum, d_coff, d_cfirst, d_cmid, d_clast, nc, d_corg, d_cbox,
                                                               haveOrigin ? 1 : 0, setOrigin ? 1 : 0, d_cre2, d_crg2, d_ccom, d_cout);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, d_cout, 12 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (setOrigin) haveOrigin = true;
    }

    void readback()
    {
        if (!initialized) throw std::runtime_error("initialize must be called first");
        if (hostPosValid) return;
        const int blocks = (int)std::min<uint32_t>((npad + kThreads - 1) / kThreads, 148 * 16);
        k_unpack<<<blocks, kThreads, 0, stream>>>(d_pos, d_img, d_s2o, npad, (int32_t)L[0], (int32_t)L[1], (int32_t)L[2], d_out);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h_out, d_out, 3 * (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        hostPosValid = true;
    }

    /* the unfolded positions straight into a caller's page-locked buffer:
     * one unpack kernel and one device-to-host copy, no pass through the
     * engine's own staging buffer (which stays as it was) */
    void readbackTo(int32_t *dst)
    {
        if (!initialized) throw std::runtime_error("initialize must be called first");
        const int blocks = (int)std::min<uint32_t>((npad + kThreads - 1) / kThreads, 148 * 16);
        k_unpack<<<blocks, kThreads, 0, stream>>>(d_pos, d_img, d_s2o, npad, (int32_t)L[0], (int32_t)L[1], (int32_t)L[2], d_out);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(dst, d_out, 3 * (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }
};

/* whether host memory at p is page-locked (cudaHostAlloc'd or registered) */
static bool host_pinned(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

/* ------------------------------------------- no-allocation colour substep
 *
 * bfm_substep_noalloc runs one colour substep on device arrays owned by the
 * caller.  Its only scratch -- the target bit lattice and the per-monomer
 * check/perform hand-over flags -- lives in the file-scope device array
 * below, so the call allocates nothing.  The array is sized for lattices of
 * up to 128^3 sites and up to 262,144 monomers per substep (512 KiB, held by
 * every GPU that loads the library until the process exits).
 */
constexpr uint32_t kNoAllocMaxSites = 1u << 21;                   /* 128^3 */
constexpr uint32_t kNoAllocMaxCount = 1u << 18;                   /* monomers per call */
constexpr size_t kNoAllocTmpWords = kNoAllocMaxSites / 32;        /* 256 KiB of target bits */
constexpr size_t kNoAllocFlagWords = kNoAllocMaxCount / 4;        /* 256 KiB of flags */

template <int RNG>
__global__ void __launch_bounds__(kThreads) k_check_na(const uint32_t *__restrict__ pos, const uint32_t *__restrict__ nbr,
                                                       const uint8_t *__restrict__ deg, uint32_t npad,
                                                       const uint32_t *__restrict__ lat, uint32_t *tmp,
                                                       uint8_t *__restrict__ flags, uint32_t off, uint32_t n,
                                                       uint32_t seed, uint32_t iter, Geometry g, Bondset bonds)
{
    __shared__ uint32_t forbid[16];
    if (threadIdx.x < 16) forbid[threadIdx.x] = bonds.forbidden[threadIdx.x];
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = off + i;
        const uint32_t r0 = pos[slot];
        const int dir = direction(draw<RNG>(seed, iter, i));
        const uint32_t r1 = zstep(r0, dir, g);
        bool ok = true;
        for (uint32_t j = 0; j < deg[slot]; ++j) {
            const uint32_t code = zbond(pos[nbr[(size_t)j * npad + slot]], r1);
            if ((forbid[code >> 5] >> (code & 31u)) & 1u) {
                ok = false;
                break;
            }
        }
        if (ok) ok = !face_occupied(lat, r0, dir, g);
        if (ok) atomicOr(tmp + (r1 >> 5), 1u << (r1 & 31u));
        flags[i] = ok ? (uint8_t)(dir | 8) : (uint8_t)0;
    }
}

__global__ void __launch_bounds__(kThreads) k_perform_na(uint32_t *__restrict__ pos, int32_t *__restrict__ img, uint32_t npad,
                                                         uint32_t *lat, const uint32_t *__restrict__ tmp,
                                                         const uint8_t *__restrict__ flags, uint32_t off, uint32_t n,
                                                         Geometry g)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t f = flags[i];
        if (!(f & 8)) continue;
        const uint32_t slot = off + i;
        const uint32_t r0 = pos[slot];
        const int dir = f & 7;
        if (face_occupied(tmp, r0, dir, g)) continue;
        const uint32_t r1 = zstep(r0, dir, g);
        atomicXor(lat + (r0 >> 5), 1u << (r0 & 31u));
        atomicXor(lat + (r1 >> 5), 1u << (r1 & 31u));
        pos[slot] = r1;
        if (img) {
            const int ax = dir >> 1;
            const bool wrapped = (dir & 1) ? ((r1 & axis_mask(g, ax)) == 0) : ((r0 & axis_mask(g, ax)) == 0);
            if (wrapped) img[(size_t)ax * npad + slot] += (dir & 1) ? 1 : -1;
        }
    }
}

} // namespace

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocTmpWords + kNoAllocFlagWords];

namespace {
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[256] = {};

/* Device address of g_noalloc_scratch on the current device.  Host code
 * cannot use the array's name: on the host it is only a stand-in symbol, so
 * the address is looked up once per device, with that device current. */
int noalloc_scratch(uint32_t **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return BFM_ECUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BFM_ECUDA;
        /* With lazy module loading a kernel is loaded (which may allocate and
         * synchronize) at its first launch.  Load all three kernels now, so
         * that no later call, whatever its RNG, loads anything. */
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k_check_na<RNG_SARU>) != cudaSuccess ||
            cudaFuncGetAttributes(&fa, k_check_na<RNG_INTHASH>) != cudaSuccess ||
            cudaFuncGetAttributes(&fa, k_perform_na) != cudaSuccess)
            return BFM_ECUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<uint32_t *>(g_noalloc_ptr[dev]);
    return BFM_OK;
}

} // namespace

struct bfm_handle {
    Engine e;
};

/* ================================================================ C ABI */

#define GUARD(h, ...)                                                 \
    do {                                                               \
        if (!(h)) return BFM_EINVAL;                                   \
        try {                                                          \
            __VA_ARGS__;                                               \
            return BFM_OK;                                             \
        } catch (CudaError const &ex) {                                \
            (h)->e.err = ex.what();                                    \
            return BFM_ECUDA;                                          \
        } catch (DeviceTimeout const &ex) {                            \
            (h)->e.err = ex.what();                                    \
            return BFM_ETIMEOUT;                                       \
        } catch (std::invalid_argument const &ex) {                    \
            (h)->e.err = ex.what();                                    \
            return BFM_EINVAL;                                         \
        } catch (std::exception const &ex) {                           \
            (h)->e.err = ex.what();                                    \
            return BFM_ERUNTIME;                                       \
        }                                                              \
    } while (0)

extern "C" {

int bfm_barrier_selftest_variant(int gpu, uint32_t timeout_ms, uint32_t extra_arrivals, uint32_t rounds, int counting,
                                 uint32_t ctas_per_sm, double *elapsed_ms);

int bfm_create(bfm_handle **out)
{
    if (!out) return BFM_EINVAL;
    try {
        auto *h = new bfm_handle();
        std::memset(h->e.forbidden, 1, sizeof(h->e.forbidden));
        *out = h;
        return BFM_OK;
    } catch (...) {
        return BFM_ERUNTIME;
    }
}

int bfm_destroy(bfm_handle *h)
{
    delete h;
    return BFM_OK;
}

const char *bfm_last_error(const bfm_handle *h) { return h ? h->e.err.c_str() : "null handle"; }

int bfm_set_gpu(bfm_handle *h, int gpu)
{
    GUARD(h, {
        int count = 0;
        CK(cudaGetDeviceCount(&count));
        if (gpu < 0 || gpu >= count)
            throw InvalidArgument("GPU with ID " + std::to_string(gpu) + " not present. Only " + std::to_string(count) + " GPUs are available.");
        CK(cudaSetDevice(gpu));
        h->e.gpu = gpu;
    });
}

int bfm_copy_bond_set(bfm_handle *h, int dx, int dy, int dz, int forbidden)
{
    GUARD(h, {
        if (dx < -4 || dx > 4 || dy < -4 || dy > 4 || dz < -4 || dz > 4) throw InvalidArgument("bond vector component outside [-4,4]");
        h->e.forbidden[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)] = forbidden ? 1 : 0;
    });
}

int bfm_set_nr_of_all_monomers(bfm_handle *h, uint32_t n)
{
    GUARD(h, {
        if (h->e.nSet) throw std::runtime_error("Number of Monomers already set to " + std::to_string(h->e.n) + "!");
        h->e.n = n;
        h->e.nSet = true;
        h->e.xyz.assign(3 * (size_t)n, 0);
        h->e.attr.assign(n, 0);
        h->e.deg.assign(n, 0);
        h->e.nbr.assign((size_t)n * 8, 0);
    });
}

int bfm_set_attribute(bfm_handle *h, uint32_t i, int32_t a)
{
    GUARD(h, {
        h->e.requireN(i);
        h->e.attr[i] = a;
    });
}

int bfm_set_monomer_coordinates(bfm_handle *h, uint32_t i, int32_t x, int32_t y, int32_t z)
{
    GUARD(h, {
        h->e.requireN(i);
        h->e.xyz[3 * (size_t)i] = x;
        h->e.xyz[3 * (size_t)i + 1] = y;
        h->e.xyz[3 * (size_t)i + 2] = z;
    });
}

int bfm_set_connectivity(bfm_handle *h, uint32_t i, uint32_t j)
{
    GUARD(h, {
        h->e.requireN(i);
        if (h->e.deg[i] >= 8) throw InvalidArgument("The maximum amount of bonds per monomer (8) has been exceeded!");
        h->e.nbr[(size_t)i * 8 + h->e.deg[i]++] = j;
    });
}

int bfm_set_lattice_size(bfm_handle *h, uint64_t bx, uint64_t by, uint64_t bz)
{
    GUARD(h, {
        const uint64_t b[3] = {bx, by, bz};
        for (int a = 0; a < 3; ++a)
            if (b[a] < 8 || b[a] > 1024 || (b[a] & (b[a] - 1)))
                throw std::runtime_error("box size must be a power of two between 8 and 1024 in each direction, got " + std::to_string(b[a]));
        for (int a = 0; a < 3; ++a) h->e.L[a] = b[a];
    });
}

int bfm_set_periodicity(bfm_handle *h, int px, int py, int pz)
{
    GUARD(h, {
        h->e.periodic[0] = px != 0;
        h->e.periodic[1] = py != 0;
        h->e.periodic[2] = pz != 0;
    });
}

int bfm_set_age(bfm_handle *h, int64_t age) { GUARD(h, { h->e.age = age; }); }
int bfm_get_age(const bfm_handle *h, int64_t *age)
{
    if (!h || !age) return BFM_EINVAL;
    *age = h->e.age;
    return BFM_OK;
}
int bfm_set_rng(bfm_handle *h, int rng)
{
    GUARD(h, {
        if (rng < 1 || rng > 5) throw InvalidArgument("unknown random number generator " + std::to_string(rng));
        h->e.rng = rng;
    });
}
int bfm_get_rng(const bfm_handle *h, int *rng)
{
    if (!h || !rng) return BFM_EINVAL;
    *rng = h->e.rng;
    return BFM_OK;
}
int bfm_set_steps_between_sortings(bfm_handle *h, int64_t steps)
{
    GUARD(h, {
        if (steps <= 0) throw InvalidArgument("steps between sortings must be positive");
        h->e.sortEvery = steps;
    });
}

int bfm_set_all_coordinates(bfm_handle *h, const int32_t *xyz, size_t n)
{
    GUARD(h, {
        if (!h->e.nSet || n != h->e.n || !xyz) throw InvalidArgument("coordinate array does not match setNrOfAllMonomers");
        std::memcpy(h->e.xyz.data(), xyz, 3 * n * sizeof(int32_t));
    });
}

int bfm_set_all_connectivity(bfm_handle *h, const uint8_t *deg, const uint32_t *nbr8, size_t n)
{
    GUARD(h, {
        if (!h->e.nSet || n != h->e.n || !deg || !nbr8) throw InvalidArgument("connectivity arrays do not match setNrOfAllMonomers");
        for (size_t i = 0; i < n; ++i)
            if (deg[i] > 8) throw InvalidArgument("The maximum amount of bonds per monomer (8) has been exceeded!");
        std::memcpy(h->e.deg.data(), deg, n);
        std::memcpy(h->e.nbr.data(), nbr8, n * 8 * sizeof(uint32_t));
    });
}

int bfm_initialize(bfm_handle *h)
{
    if (!h) return BFM_EINVAL;
    try {
        h->e.initialize();
        return BFM_OK;
    } catch (CudaError const &ex) {
        h->e.err = ex.what();
        h->e.release();
        return BFM_ECUDA;
    } catch (std::invalid_argument const &ex) {
        h->e.err = ex.what();
        h->e.release();
        return BFM_EINVAL;
    } catch (std::exception const &ex) {
        h->e.err = ex.what();
        h->e.release();
        return BFM_ERUNTIME;
    }
}

int bfm_run(bfm_handle *h, uint32_t nmcs)
{
    if (h && !h->e.initialized) {
        h->e.err = "initialize must be called before runSimulationOnGPU";
        return BFM_ENOTINIT;
    }
    GUARD(h, { h->e.run(nmcs); });
}

int bfm_get_monomer_position(bfm_handle *h, uint32_t i, int32_t *x, int32_t *y, int32_t *z)
{
    if (h && !h->e.initialized) {
        h->e.err = "initialize must be called first";
        return BFM_ENOTINIT;
    }
    GUARD(h, {
        h->e.requireN(i);
        h->e.readback();
        if (x) *x = h->e.h_out[3 * (size_t)i];
        if (y) *y = h->e.h_out[3 * (size_t)i + 1];
        if (z) *z = h->e.h_out[3 * (size_t)i + 2];
    });
}

int bfm_get_positions(bfm_handle *h, int32_t *xyz, size_t n)
{
    if (h && !h->e.initialized) {
        h->e.err = "initialize must be called first";
        return BFM_ENOTINIT;
    }
    GUARD(h, {
        if (!xyz || n != h->e.n) throw InvalidArgument("position buffer does not match the number of monomers");
        if (!h->e.hostPosValid && host_pinned(xyz)) {
            h->e.readbackTo(xyz);
        } else {
            h->e.readback();
            std::memcpy(xyz, h->e.h_out, 3 * n * sizeof(int32_t));
        }
    });
}

int bfm_analyzer_init(bfm_handle *h, uint32_t *n_chains)
{
    if (h && !h->e.initialized) {
        h->e.err = "initialize must be called first";
        return BFM_ENOTINIT;
    }
    GUARD(h, {
        h->e.analyzerInit();
        if (n_chains) *n_chains = h->e.nChains();
    });
}

int bfm_analyze(bfm_handle *h, int set_origin, double *out, size_t n_out)
{
    if (h && !h->e.initialized) {
        h->e.err = "initialize must be called first";
        return BFM_ENOTINIT;
    }
    GUARD(h, {
        if (!out || n_out < 11) throw InvalidArgument("bfm_analyze needs an output array of at least 11 doubles");
        double tmp[12];
        h->e.analyze(tmp, set_origin != 0);
        std::memcpy(out, tmp, (n_out < 12 ? 11 : 12) * sizeof(double));
    });
}

int bfm_analyzer_chain_ids(bfm_handle *h, uint32_t *first, uint32_t *middle, uint32_t *last, uint32_t n_chains)
{
    GUARD(h, {
        if (!h->e.chainsReady) throw std::runtime_error("bfm_analyzer_init must be called first");
        if (n_chains != h->e.nChains()) throw InvalidArgument("n_chains does not match the number of chains");
        if (first) std::memcpy(first, h->e.chains.first.data(), n_chains * sizeof(uint32_t));
        if (middle) std::memcpy(middle, h->e.chains.middle.data(), n_chains * sizeof(uint32_t));
        if (last) std::memcpy(last, h->e.chains.last.data(), n_chains * sizeof(uint32_t));
    });
}

int bfm_analyze_per_chain(bfm_handle *h, double *re2, double *rg2, double *com, uint32_t n_chains)
{
    GUARD(h, {
        if (!h->e.chainsReady) throw std::runtime_error("bfm_analyzer_init must be called first");
        if (n_chains != h->e.nChains()) throw InvalidArgument("n_chains does not match the number of chains");
        auto &e = h->e;
        if (re2) CK(cudaMemcpyAsync(re2, e.d_cre2, n_chains * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        if (rg2) CK(cudaMemcpyAsync(rg2, e.d_crg2, n_chains * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        if (com) CK(cudaMemcpyAsync(com, e.d_ccom, 3 * (size_t)n_chains * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        CK(cudaStreamSynchronize(e.stream));
    });
}

int bfm_set_filter_stats(bfm_handle *h, int mode)
{
    GUARD(h, {
        if (mode < 0 || mode > 2) throw std::invalid_argument("filter statistics mode must be 0, 1 or 2");
        h->e.filterStats = mode;
    });
}

int bfm_get_filter_stats(const bfm_handle *h, double *out, size_t n_out)
{
    if (!h || !out) return BFM_EINVAL;
    if (!h->e.initialized) return BFM_ENOTINIT;
    const auto &e = h->e;
    const size_t z = (size_t)e.nSpecies * kFilters;
    if (n_out < 5 * z) return BFM_EINVAL;
    for (size_t i = 0; i < z; ++i) {
        const double n = i < e.fcnt.size() ? e.fcnt[i] : 0.0;
        double *o = out + 5 * i;
        o[4] = n;
        if (n == 0.0) {
            o[0] = o[1] = o[2] = o[3] = 0.0;
            continue;
        }
        const double mean = e.fsum[i] / n, sum2 = e.fsum2[i] / n;
        o[0] = e.fmin[i];
        o[1] = mean;
        o[2] = std::sqrt(n / (n - 1.0) * (sum2 - mean * mean)); /* .cu:3363-3366; NaN when n == 1 */
        o[3] = e.fmax[i];
    }
    return BFM_OK;
}

int bfm_cleanup(bfm_handle *h)
{
    GUARD(h, {
        h->e.release();
        h->e.nSet = false;
        h->e.n = 0;
    });
}

int bfm_get_lattice_words(const bfm_handle *h, size_t *nwords)
{
    if (!h || !nwords) return BFM_EINVAL;
    if (!h->e.initialized) return BFM_ENOTINIT;
    *nwords = h->e.latWords;
    return BFM_OK;
}

int bfm_get_lattice(bfm_handle *h, uint32_t *words, size_t nwords)
{
    if (h && !h->e.initialized) return BFM_ENOTINIT;
    GUARD(h, {
        if (!words || nwords != h->e.latWords) throw InvalidArgument("lattice buffer size mismatch");
        CK(cudaMemcpyAsync(words, h->e.d_lat, nwords * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->e.stream));
        CK(cudaStreamSynchronize(h->e.stream));
    });
}

int bfm_get_nspecies(const bfm_handle *h, uint32_t *ns)
{
    if (!h || !ns) return BFM_EINVAL;
    if (!h->e.initialized) return BFM_ENOTINIT;
    *ns = h->e.nSpecies;
    return BFM_OK;
}

int bfm_get_colors(const bfm_handle *h, uint32_t *colors, size_t n)
{
    if (!h || !colors) return BFM_EINVAL;
    if (!h->e.initialized) return BFM_ENOTINIT;
    if (n != h->e.n) return BFM_EINVAL;
    std::memcpy(colors, h->e.color.data(), n * sizeof(uint32_t));
    return BFM_OK;
}

int bfm_get_species_order(bfm_handle *h, uint32_t sp, uint32_t *ids, size_t cap, size_t *count)
{
    if (h && !h->e.initialized) return BFM_ENOTINIT;
    GUARD(h, {
        if (sp >= h->e.nSpecies) throw InvalidArgument("species index out of range");
        const Species s = h->e.spec[sp];
        if (count) *count = s.n;
        if (ids) {
            if (cap < s.n) throw InvalidArgument("buffer too small");
            CK(cudaMemcpyAsync(ids, h->e.d_s2o + s.off, s.n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->e.stream));
            CK(cudaStreamSynchronize(h->e.stream));
        }
    });
}

int bfm_get_counters(bfm_handle *h, uint64_t out3[3])
{
    if (h && !h->e.initialized) return BFM_ENOTINIT;
    GUARD(h, {
        unsigned long long c[4];
        CK(cudaMemcpyAsync(c, h->e.d_counters, sizeof(c), cudaMemcpyDeviceToHost, h->e.stream));
        CK(cudaStreamSynchronize(h->e.stream));
        out3[0] = h->e.nAttempts;
        out3[1] = c[0];
        out3[2] = c[1];
    });
}

int bfm_get_last_run_ms(const bfm_handle *h, double *ms)
{
    if (!h || !ms) return BFM_EINVAL;
    *ms = h->e.lastRunMs;
    return BFM_OK;
}

int bfm_get_last_run_launches(const bfm_handle *h, uint64_t *launches)
{
    if (!h || !launches) return BFM_EINVAL;
    *launches = h->e.lastLaunches;
    return BFM_OK;
}

int bfm_time_kernels(bfm_handle *h, uint32_t nmcs, double *ms, uint64_t *launches, uint64_t *attempts)
{
    if (h && !h->e.initialized) return BFM_ENOTINIT;
    GUARD(h, {
        if (!ms || !launches || !attempts) throw InvalidArgument("null output pointer");
        h->e.timeKernels(nmcs, ms, launches, attempts);
    });
}

int bfm_set_sweep_shape(bfm_handle *h, int shape)
{
    GUARD(h, {
        if (shape < -1 || shape > 10) throw InvalidArgument("sweep shape must be -1 (automatic) or 0..10");
        h->e.forcedShape = shape;
        if (h->e.initialized) h->e.configureSweep();
    });
}

int bfm_set_sweep_autotune(bfm_handle *h, int on)
{
    GUARD(h, {
        h->e.autotune = on != 0;
        h->e.tuned = false;
    });
}

int bfm_get_sweep_tuning(const bfm_handle *h, int *tuned, uint32_t *count, int *shapes, int *extra_rounds, int *threads,
                         double *ns_per_move, uint32_t cap)
{
    if (!h) return BFM_EINVAL;
    const auto &t = h->e.trials;
    if (tuned) *tuned = h->e.tuned ? 1 : 0;
    if (count) *count = (uint32_t)t.size();
    for (uint32_t i = 0; i < t.size() && i < cap; ++i) {
        if (shapes) shapes[i] = t[i].shape;
        if (extra_rounds) extra_rounds[i] = t[i].extra;
        if (threads) threads[i] = t[i].threads;
        if (ns_per_move) ns_per_move[i] = t[i].nsPerMove;
    }
    return BFM_OK;
}

int bfm_get_launch_info(const bfm_handle *h, int *mode, int *grid, int *threads, size_t *smem_bytes)
{
    if (!h) return BFM_EINVAL;
    if (!h->e.initialized) return BFM_ENOTINIT;
    if (mode) *mode = h->e.launchMode == 0 ? h->e.sweepMode : -h->e.launchMode;
    if (grid) *grid = h->e.sweepGrid;
    if (threads) *threads = h->e.sweepThreads;
    if (smem_bytes) *smem_bytes = h->e.sweepSmem;
    return BFM_OK;
}

int bfm_set_barrier_timeout_ms(bfm_handle *h, uint32_t ms)
{
    GUARD(h, {
        if (ms == 0) throw InvalidArgument("barrier timeout must be positive");
        h->e.timeoutNs = (unsigned long long)ms * 1000000ull;
    });
}

int bfm_barrier_selftest(int gpu, uint32_t timeout_ms, uint32_t extra_arrivals, uint32_t rounds, double *elapsed_ms)
{
    return bfm_barrier_selftest_variant(gpu, timeout_ms, extra_arrivals, rounds, 1, 0, elapsed_ms);
}

int bfm_barrier_selftest_variant(int gpu, uint32_t timeout_ms, uint32_t extra_arrivals, uint32_t rounds, int counting,
                                 uint32_t ctas_per_sm, double *elapsed_ms)
{
    GridBarrier *bar = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int status = BFM_OK;
    do {
        if (cudaSetDevice(gpu) != cudaSuccess) { status = BFM_ECUDA; break; }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu) != cudaSuccess) { status = BFM_ECUDA; break; }
        if (cudaMalloc((void **)&bar, sizeof(GridBarrier)) != cudaSuccess) { status = BFM_ECUDA; break; }
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { status = BFM_ECUDA; break; }
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaMemsetAsync(bar, 0, sizeof(GridBarrier), st);
        const unsigned int grid = (unsigned int)sms * (ctas_per_sm ? ctas_per_sm : 1u);
        unsigned int expected = grid + extra_arrivals;
        unsigned long long to = (unsigned long long)timeout_ms * 1000000ull;
        void *args[] = {&bar, &expected, &to, &rounds, &counting};
        cudaEventRecord(e0, st);
        if (cudaLaunchCooperativeKernel((const void *)k_barrier_selftest, dim3(grid), dim3(64), args, 0, st) != cudaSuccess) {
            status = BFM_ECUDA;
            break;
        }
        cudaEventRecord(e1, st);
        GridBarrier hb;
        if (cudaMemcpyAsync(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            status = BFM_ECUDA;
            break;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (elapsed_ms) *elapsed_ms = ms;
        status = hb.err ? BFM_ETIMEOUT : BFM_OK;
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (bar) cudaFree(bar);
    return status;
}

int bfm_set_launch_mode(bfm_handle *h, int mode)
{
    GUARD(h, {
        if (mode < 0 || mode > 2) throw InvalidArgument("launch mode must be 0 (persistent), 1 (graphs) or 2 (direct)");
        h->e.launchMode = mode;
    });
}

int bfm_set_coloring(bfm_handle *h, int mode)
{
    GUARD(h, {
        if (mode != 0 && mode != 1) throw InvalidArgument("colouring mode must be 0 (host) or 1 (device)");
        h->e.coloringMode = mode;
    });
}

int bfm_get_coloring(const bfm_handle *h, int *mode, int *on_device)
{
    if (!h) return BFM_EINVAL;
    if (mode) *mode = h->e.coloringMode;
    if (on_device) *on_device = h->e.colorOnDevice;
    return BFM_OK;
}

int bfm_color_graph_device(int gpu, uint32_t n, const uint8_t *deg, const uint32_t *nbr8, int uniform, uint32_t *colors,
                           uint32_t *ncolors, int *on_device)
{
    if ((n && (!deg || !nbr8 || !colors)) || !ncolors) return BFM_EINVAL;
    try {
        for (uint32_t i = 0; i < n; ++i) {
            if (deg[i] > 8) return BFM_EINVAL;
            for (uint32_t j = 0; j < deg[i]; ++j)
                if (nbr8[(size_t)i * 8 + j] >= n) return BFM_EINVAL;
        }
        if (cudaSetDevice(gpu) != cudaSuccess) return BFM_ECUDA;
        std::vector<uint32_t> c;
        const int dev = color_graph_device(n, deg, nbr8, uniform != 0, c);
        if (!dev) c = color_graph(n, deg, nbr8, uniform != 0);
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            colors[i] = c[i];
            k = std::max(k, c[i] + 1);
        }
        *ncolors = k;
        if (on_device) *on_device = dev;
        return BFM_OK;
    } catch (std::exception const &) {
        return BFM_ECUDA;
    }
}

int bfm_color_graph(uint32_t n, const uint8_t *deg, const uint32_t *nbr8, int uniform, uint32_t *colors, uint32_t *ncolors)
{
    if ((n && (!deg || !nbr8 || !colors)) || !ncolors) return BFM_EINVAL;
    try {
        for (uint32_t i = 0; i < n; ++i) {
            if (deg[i] > 8) return BFM_EINVAL;
            for (uint32_t j = 0; j < deg[i]; ++j)
                if (nbr8[(size_t)i * 8 + j] >= n) return BFM_EINVAL;
        }
        const std::vector<uint32_t> c = color_graph(n, deg, nbr8, uniform != 0);
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            colors[i] = c[i];
            k = std::max(k, c[i] + 1);
        }
        *ncolors = k;
        return BFM_OK;
    } catch (...) {
        return BFM_ERUNTIME;
    }
}

int bfm_substep_noalloc(uint32_t *pos, int32_t *img, const uint32_t *nbr, const uint8_t *deg, uint32_t npad,
                        uint32_t *lattice, uint32_t box_x, uint32_t box_y, uint32_t box_z, const uint8_t *allowed512,
                        uint32_t slot_offset, uint32_t count, uint32_t seed, uint32_t iteration, int rng, void *stream)
{
    if (!pos || !nbr || !deg || !lattice || !allowed512) return BFM_EINVAL;
    if (rng != BFM_RNG_INTHASH && rng != BFM_RNG_SARU) return BFM_EINVAL;
    /* an error left pending by the caller's own earlier work stays theirs:
     * nothing runs, and it is not cleared */
    if (cudaPeekAtLastError() != cudaSuccess) return BFM_ECUDA;
    const uint32_t b[3] = {box_x, box_y, box_z};
    uint32_t Lm = 0;
    for (int a = 0; a < 3; ++a) {
        if (b[a] < 8 || (b[a] & (b[a] - 1))) return BFM_EINVAL;
        Lm = std::max(Lm, b[a]);
    }
    if ((uint64_t)Lm * Lm * Lm > kNoAllocMaxSites || count > kNoAllocMaxCount) return BFM_ETOOLARGE;
    if ((uint64_t)slot_offset + count > npad) return BFM_EINVAL;
    unsigned nAllowed = 0;
    Bondset bonds;
    std::memset(&bonds, 0, sizeof(bonds));
    for (uint32_t dz = 0; dz < 8; ++dz)
        for (uint32_t dy = 0; dy < 8; ++dy)
            for (uint32_t dx = 0; dx < 8; ++dx) {
                if (allowed512[dx | (dy << 3) | (dz << 6)]) {
                    ++nAllowed;
                } else {
                    const uint32_t code = zcode(dx, dy, dz);
                    bonds.forbidden[code >> 5] |= 1u << (code & 31);
                }
            }
    if (nAllowed != 108) return BFM_EINVAL;
    Geometry g;
    for (int a = 0; a < 3; ++a) g.m[a] = dilate3(b[a] - 1) << a;
    uint32_t *scratch = nullptr;
    const int st = noalloc_scratch(&scratch);
    if (st != BFM_OK) return st;
    uint32_t *tmp = scratch;
    uint8_t *flags = reinterpret_cast<uint8_t *>(scratch + kNoAllocTmpWords);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t words = (size_t)Lm * Lm * Lm / 32;
    if (cudaMemsetAsync(tmp, 0, words * sizeof(uint32_t), s) != cudaSuccess) return BFM_ECUDA;
    if (count) {
        const int blocks = (int)std::min<uint32_t>((count + kThreads - 1) / kThreads, 148u * 16u);
        if (rng == BFM_RNG_SARU)
            k_check_na<RNG_SARU><<<blocks, kThreads, 0, s>>>(pos, nbr, deg, npad, lattice, tmp, flags, slot_offset, count, seed, iteration, g, bonds);
        else
            k_check_na<RNG_INTHASH><<<blocks, kThreads, 0, s>>>(pos, nbr, deg, npad, lattice, tmp, flags, slot_offset, count, seed, iteration, g, bonds);
        k_perform_na<<<blocks, kThreads, 0, s>>>(pos, img, npad, lattice, tmp, flags, slot_offset, count, g);
    }
    return cudaGetLastError() == cudaSuccess ? BFM_OK : BFM_ECUDA;
}

int bfm_r250_seed(uint64_t seed)
{
    std::lock_guard<std::mutex> lock(g_r250_mutex);
    global_r250().seed_u64(seed);
    return BFM_OK;
}

int bfm_r250_seed_words(const uint32_t *words, size_t n)
{
    if (!words || n < 250) return BFM_EINVAL;
    std::lock_guard<std::mutex> lock(g_r250_mutex);
    global_r250().seed_words(words);
    return BFM_OK;
}

int bfm_r250_get_state(uint32_t state251[251])
{
    if (!state251) return BFM_EINVAL;
    std::lock_guard<std::mutex> lock(g_r250_mutex);
    std::memcpy(state251, global_r250().buf, 250 * sizeof(uint32_t));
    state251[250] = global_r250().idx;
    return BFM_OK;
}

int bfm_r250_set_state(const uint32_t state251[251])
{
    if (!state251 || state251[250] >= 250) return BFM_EINVAL;
    std::lock_guard<std::mutex> lock(g_r250_mutex);
    std::memcpy(global_r250().buf, state251, 250 * sizeof(uint32_t));
    global_r250().idx = state251[250];
    return BFM_OK;
}

uint32_t bfm_r250_rand32(void)
{
    std::lock_guard<std::mutex> lock(g_r250_mutex);
    return global_r250().next();
}

} /* extern "C" */
