/*
 * bfm_sweep.cuh -- the persistent colour-substep kernel.
 *
 * One cooperative launch runs a chunk of colour substeps.  Per substep:
 *
 *   phase A (check)    every monomer of the colour draws its move, tests its
 *                      bonds and the leading face on the occupation lattice,
 *                      and -- if both pass -- marks its target in the
 *                      substep's target lattice and appends itself to its
 *                      CTA's candidate list;
 *   grid barrier
 *   phase B (perform)  each CTA walks only its own candidates: a candidate
 *                      moves unless another candidate's target lies in its
 *                      leading face (the reference's deterministic two-phase
 *                      rule, UpdaterGPUScBFM_AB_Type.cu:1148-1190);
 *   grid barrier
 *
 * and at the start of the next substep each CTA zeroes the target words of
 * its previous candidates (the target lattice is double buffered, so this
 * never races with the marks of the running substep).  Lattices are read as
 * 64-bit words: a word is a 4x4x4 brick of sites in Z-order, so the nine
 * sites of a leading face lie in at most four words (face_words), whose
 * masks come from a table in shared memory (face_table_entry).
 *
 * Grid barriers wait with a bound: after `timeoutNs` of %globaltimer (or a
 * fixed number of polls) a waiting CTA raises the error word and every CTA
 * leaves the kernel, so a broken launch ends with BFM_ETIMEOUT instead of a
 * hang.
 */
#pragma once
#include <cstdint>

#include "bfm_device.cuh"

namespace bfm {

struct GridBarrier {
    unsigned int count; /* CTAs arrived at the current barrier */
    unsigned int gen;   /* barrier generation, bumped by the last arrival */
    unsigned int err;   /* non-zero: a wait timed out, leave the kernel */
    unsigned int pad;
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned int kBarrierMaxPolls = 1u << 26;

/* Grid-wide barrier for co-resident CTAs (cooperative launch).  `gen` is the
 * generation the calling CTA expects (kept by thread 0).  Returns false on
 * all threads of the CTA when the barrier failed (timeout here or elsewhere). */
__device__ __forceinline__ bool grid_barrier(GridBarrier *bar, unsigned int nblocks, unsigned int &gen,
                                             unsigned long long timeoutNs)
{
    __shared__ unsigned int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ok = 1;
        __threadfence();
        const unsigned int arrived = atomicAdd(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicExch(&bar->gen, gen + 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned int polls = 0;
            while (ld_acquire_gpu(&bar->gen) == gen) {
                if (ld_acquire_gpu(&bar->err)) {
                    ok = 0;
                    break;
                }
                if (++polls > kBarrierMaxPolls || global_ns() - t0 > timeoutNs) {
                    atomicExch(&bar->err, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        gen += 1u;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

/* Counting grid barrier: the counter only grows.  Each CTA adds 1 with a
 * release reduction (no return value, nothing to wait for) and then waits
 * until the counter reaches `target` = (barriers passed so far + 1) x CTAs,
 * reading it with acquire semantics.  The counter starts at 0 for every
 * launch (the host clears it before the launch). */
__device__ __forceinline__ void red_release_add(unsigned int *p, unsigned int v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_barrier_count(GridBarrier *bar, unsigned int &target, unsigned int nblocks,
                                                   unsigned long long timeoutNs)
{
    __shared__ unsigned int s_ok2;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ok = 1;
        target += nblocks;
        red_release_add(&bar->count, 1u);
        const unsigned long long t0 = global_ns();
        unsigned int polls = 0;
        while ((int)(ld_acquire_gpu(&bar->count) - target) < 0) {
            if (ld_acquire_gpu(&bar->err)) {
                ok = 0;
                break;
            }
            if (++polls > kBarrierMaxPolls || global_ns() - t0 > timeoutNs) {
                atomicExch(&bar->err, 1u);
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
        s_ok2 = ok;
    }
    __syncthreads();
    return s_ok2 != 0;
}

/* Split form of the counting barrier, so that a CTA can do work that does
 * not depend on the other CTAs between its arrival and its wait.
 * grid_arrive: after a __syncthreads that ends the CTA's part, thread 0 adds
 * its arrival with release semantics.  grid_wait: thread 0 polls the counter
 * (acquire) until `target` arrivals; the error word and the clock are read
 * only every 32 polls so that a poll is a single load.  Both return the
 * CTA-wide verdict through shared memory after a __syncthreads. */
__device__ __forceinline__ void grid_arrive(GridBarrier *bar, unsigned int &target, unsigned int nblocks)
{
    if (threadIdx.x == 0) {
        target += nblocks;
        red_release_add(&bar->count, 1u);
    }
}

__device__ __forceinline__ bool grid_wait(GridBarrier *bar, unsigned int target, unsigned long long timeoutNs)
{
    __shared__ unsigned int s_ok3;
    if (threadIdx.x == 0) {
        unsigned int ok = 1;
        if ((int)(ld_acquire_gpu(&bar->count) - target) < 0) {
            const unsigned long long t0 = global_ns();
            for (unsigned int polls = 1;; ++polls) {
                if ((int)(ld_acquire_gpu(&bar->count) - target) >= 0) break;
                if ((polls & 31u) == 0) {
                    if (ld_acquire_gpu(&bar->err)) {
                        ok = 0;
                        break;
                    }
                    if (polls > kBarrierMaxPolls || global_ns() - t0 > timeoutNs) {
                        atomicExch(&bar->err, 1u);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok3 = ok;
    }
    __syncthreads();
    return s_ok3 != 0;
}

/* ---- bulk (TMA) copies global -> shared on an mbarrier ------------------ */

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

/* 1-D bulk copy: dst, src 16-byte aligned, bytes a multiple of 16 */
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

/* generic-proxy accesses before, async-proxy (bulk copy) accesses after */
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

/* wait for the phase `parity` of the mbarrier with a bound; false on timeout */
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t parity, unsigned long long timeoutNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned int polls = 0; polls < kBarrierMaxPolls; ++polls) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > timeoutNs) return false;
    }
    return false;
}

/* Per-direction constants: payload masks of the move axis and of the two
 * transverse axes, their unit bits, and the bit position of the transverse
 * axes (for extracting their two low coordinate bits). */
struct DirConst {
    uint32_t ma, mb, mc, ua;
    uint32_t ub, uc, bx, cx;
};

__device__ __forceinline__ void build_dir_table(DirConst *t, const Geometry &g)
{
    if (threadIdx.x < 6) {
        const int dir = threadIdx.x, ax = dir >> 1;
        const int bx = (ax == 0) ? 1 : 0;
        const int cx = (ax == 2) ? 1 : 2;
        DirConst d;
        d.ma = axis_mask(g, ax);
        d.mb = axis_mask(g, bx);
        d.mc = axis_mask(g, cx);
        d.ua = 1u << ax;
        d.ub = 1u << bx;
        d.uc = 1u << cx;
        d.bx = (uint32_t)bx;
        d.cx = (uint32_t)cx;
        t[dir] = d;
    }
}

/* Unit step along the move axis of dir, using the per-direction constants. */
__device__ __forceinline__ uint32_t dstep(uint32_t a, int dir, const DirConst &d)
{
    return (dir & 1) ? ((a & ~d.ma) | (((a | ~d.ma) + d.ua) & d.ma)) : ((a & ~d.ma) | (((a & d.ma) - d.ua) & d.ma));
}

} // namespace bfm
