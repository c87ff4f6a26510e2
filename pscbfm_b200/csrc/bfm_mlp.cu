/*
 * bfm_mlp.cu -- the small multilayer perceptron of the learned run schedule:
 * in -> 128 -> 128 -> out (ReLU), trained and evaluated on the GPU by one
 * kernel of this file on the fifth-generation tensor cores.
 *
 * k_mlp runs whole training steps in one cooperative launch: per step, each
 * CTA takes 128-row tiles of the batch (one thread per row), and every
 * product of the forward and backward passes is a tcgen05.mma of M = 128
 * rows with bf16 operands in shared memory and an fp32 accumulator in tensor
 * memory (TMEM), issued by one thread and completed through an mbarrier:
 *
 *   forward   Z1 = X W1^T, Z2 = H1 W2^T, Y = H2 W3^T          (rows x features)
 *   backward  dH2 = dY W3, dH1 = dZ2 W2                        (rows x features)
 *             dW3^T = H2^T dY, dW2 = dZ2^T H1, dW1 = dZ1^T X  (features x features,
 *             accumulated over the CTA's tiles in TMEM)
 *
 * The epilogues read the accumulators row by row (tcgen05.ld, 32 lanes per
 * warp), add biases, apply ReLU and its derivative, round to bf16 and store
 * the next operand.  Every bf16 matrix lives in shared memory in one layout,
 * "column planes": element (r, c) of an R-row matrix at byte
 * ((c / 8) * R + r) * 16 + (c % 8) * 2, i.e. 8 x 8 core matrices of 16-byte
 * rows, so the same buffer is a K-major operand (rows = M or N) and an
 * MN-major operand (rows = K) of the canonical no-swizzle layout; only the
 * descriptor's leading and stride byte offsets differ.  The per-CTA weight
 * gradients go to global memory; after a grid barrier every parameter's
 * gradient is summed over the CTAs in a fixed order (deterministic), Adam
 * updates the fp32 masters, and after a second barrier the next step loads
 * the updated weights (rounded to bf16) into shared memory.
 *
 * Rounding points (the oracle, oracle/mlp_oracle.py, uses the same): inputs,
 * weights, hidden activations and the backward signals dY, dZ2, dZ1 are
 * rounded to bf16 for the products; biases, accumulators, bias gradients,
 * the loss and Adam are fp32.
 *
 * Not in the reference: it feeds the batched ensembles' schedule
 * (per-system MCS budgets and admission order).
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfm_sweep.cuh"
#include "../../include/pscbfm_b200.h"

namespace bfm {
namespace mlp {

constexpr uint32_t kTile = 128;  /* batch rows per tile: the MMA's M */
constexpr uint32_t kH = 128;     /* hidden width */
constexpr uint32_t kIO = 16;     /* input and output widths, padded */
constexpr int kThreads = 128;    /* one thread per tile row (TMEM lane) */
constexpr uint32_t kTmemCols = 512;

/* TMEM columns: transient accumulators and the per-CTA weight gradients */
constexpr uint32_t kTA = 0;      /* Z1, then dH2 */
constexpr uint32_t kTB = 128;    /* Z2, then dH1 */
constexpr uint32_t kTW2 = 256;   /* dW2 (out x in) */
constexpr uint32_t kTC = 384;    /* Y (16 columns) */
constexpr uint32_t kTW3 = 400;   /* dW3^T (hidden x out, 16 columns) */
constexpr uint32_t kTW1 = 416;   /* dW1 (hidden x in, 16 columns) */

/* shared memory (bytes): bf16 matrices in column planes, then fp32 vectors */
constexpr uint32_t kOffW1 = 0;                          /* 128 x 16  */
constexpr uint32_t kOffW2 = kOffW1 + 128 * 16 * 2;      /* 128 x 128 */
constexpr uint32_t kOffW3 = kOffW2 + 128 * 128 * 2;     /* 16 x 128  */
constexpr uint32_t kOffX = kOffW3 + 16 * 128 * 2;       /* 128 x 16  */
constexpr uint32_t kOffH1 = kOffX + 128 * 16 * 2;       /* H1, then dZ1 */
constexpr uint32_t kOffH2 = kOffH1 + 128 * 128 * 2;     /* H2, then dZ2 */
constexpr uint32_t kOffDY = kOffH2 + 128 * 128 * 2;     /* 128 x 16  */
constexpr uint32_t kOffB = kOffDY + 128 * 16 * 2;       /* b1, b2 (128 each), b3 (16) */
constexpr uint32_t kOffDB = kOffB + (128 + 128 + 16) * 4; /* db1, db2 (128 each), db3 (32) of the step */
constexpr uint32_t kOffRed = kOffDB + (128 + 128 + 32) * 4; /* 128 x 33 fp32 transpose scratch */
constexpr uint32_t kSmemBytes = kOffRed + 128 * 33 * 4 + 64;
/* more than half of an SM's shared memory: one CTA per SM, so the 512-column
 * TMEM allocation never waits for another CTA */
static_assert(kSmemBytes > 120 * 1024 && kSmemBytes <= 227 * 1024, "shared-memory plan");

enum Mode { MODE_FORWARD = 0, MODE_GRADIENTS = 1, MODE_TRAIN = 2 };

struct Args {
    uint32_t I, O, nParam;
    uint32_t oW1, ob1, oW2, ob2, oW3, ob3;
    int mode;
    uint32_t nsteps;
    const uint32_t *stepRows; /* rows of each step */
    const uint32_t *stepOff;  /* first entry of each step in rowIdx (or in x when rowIdx is null) */
    const uint32_t *rowIdx;   /* row of x / t of each entry, or null */
    const float *x, *t, *w;
    float *y;                 /* forward: rows x O */
    float *p, *m1, *m2, *g;
    float *part;              /* grid x nParam */
    float *lossPart;          /* grid */
    float *losses;            /* per step */
    const float *c1, *c2;     /* Adam bias corrections per step */
    float lr, beta1, beta2, eps;
    GridBarrier *bar;
    unsigned long long timeoutNs;
    unsigned int *err;
};

/* ------------------------------------------------------------ PTX helpers */

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

/* shared-memory matrix descriptor of the canonical layout without swizzle
 * (tcgen05 version 1): start, leading and stride byte offsets in 16-byte units */
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

/* instruction descriptor of kind::f16: bf16 A and B, fp32 D, M = 128 */
__host__ __device__ constexpr uint32_t idesc(uint32_t N, bool aMN, bool bMN)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((aMN ? 1u : 0u) << 15) | ((bMN ? 1u : 0u) << 16) | ((N >> 3) << 17) |
           ((kTile >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
                 "l"(a), "l"(b), "r"(id), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(unsigned long long *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(mbar))
                 : "memory");
}

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* 16 consecutive fp32 columns of this thread's TMEM lane */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    tc_wait_ld();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

/* element (r, c) of an R-row bf16 matrix in column planes: byte offset */
__device__ __forceinline__ uint32_t plane_off(uint32_t R, uint32_t r, uint32_t c) { return ((c >> 3) * R + r) * 16u + (c & 7u) * 2u; }

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&v);
}

/* eight columns c8*8 .. c8*8+7 of row r as one 16-byte store */
__device__ __forceinline__ void st_row8(unsigned char *buf, uint32_t R, uint32_t r, uint32_t c8, const float *v)
{
    uint4 q;
    q.x = pack2(v[0], v[1]);
    q.y = pack2(v[2], v[3]);
    q.z = pack2(v[4], v[5]);
    q.w = pack2(v[6], v[7]);
    *reinterpret_cast<uint4 *>(buf + (c8 * R + r) * 16u) = q;
}

/* bounded wait for the completion of the thread block's latest MMA group:
 * thread 0 waits on the mbarrier, the block learns the verdict at a barrier
 * (so every thread takes the same path), and the TMEM reads that follow are
 * ordered after it */
__device__ __forceinline__ bool mma_wait(unsigned long long *mbar, uint32_t &phase, unsigned long long timeoutNs,
                                         volatile unsigned int *okFlag)
{
    if (threadIdx.x == 0 && !mbar_wait_bounded(mbar, phase, timeoutNs)) *okFlag = 0u;
    phase ^= 1u;
    __syncthreads();
    tc_after_sync();
    return *okFlag != 0u;
}

/* make this thread's shared-memory operands and TMEM reads ordered before
 * the MMAs the elected thread issues after the barrier */
__device__ __forceinline__ void before_mma()
{
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
}

/* column sums over the tile's 128 rows of 32 fp32 values per thread (this
 * thread's row), accumulated into acc[0..31], in a fixed order */
__device__ __forceinline__ void column_sums32(float *red, const float *v, float *acc)
{
    const uint32_t tid = threadIdx.x;
#pragma unroll
    for (int j = 0; j < 32; ++j) red[tid * 33 + j] = v[j];
    __syncthreads();
    if (tid < 32) {
        float s = 0.f;
        for (uint32_t r = 0; r < kTile; ++r) s += red[r * 33 + tid];
        acc[tid] += s;
    }
    __syncthreads();
}

/* ------------------------------------------------------------------ kernel */

__global__ void __launch_bounds__(kThreads, 1) k_mlp(Args a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ unsigned long long s_mbar;
    __shared__ uint32_t s_tmem;
    __shared__ float s_loss[4];
    __shared__ unsigned int s_ok;
    unsigned char *sW1 = sm + kOffW1, *sW2 = sm + kOffW2, *sW3 = sm + kOffW3, *sX = sm + kOffX;
    unsigned char *sH1 = sm + kOffH1, *sH2 = sm + kOffH2, *sDY = sm + kOffDY;
    float *sb1 = reinterpret_cast<float *>(sm + kOffB), *sb2 = sb1 + kH, *sb3 = sb2 + kH;
    float *db1 = reinterpret_cast<float *>(sm + kOffDB), *db2 = db1 + kH, *db3 = db2 + kH;
    float *red = reinterpret_cast<float *>(sm + kOffRed);

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t I = a.I, O = a.O;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_tmem)), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&s_mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tm = s_tmem;
    const uint32_t lanes = (warp * 32u) << 16; /* this warp's TMEM lanes */
    uint32_t phase = 0;
    bool ok = true;
    unsigned int target = 0;

    /* operand descriptors (column planes; see the file comment) */
    const uint32_t aW1 = saddr(sW1), aW2 = saddr(sW2), aW3 = saddr(sW3), aX = saddr(sX);
    const uint32_t aH1 = saddr(sH1), aH2 = saddr(sH2), aDY = saddr(sDY);
    /* K-major, 128 rows: 8-row groups 128 B apart, K planes 2048 B apart;
     * K-major, 16 rows: K planes 256 B apart */
    auto kmaj128 = [](uint32_t base, uint32_t k0) { return sdesc(base + (k0 >> 3) * 2048u, 2048u, 128u); };
    auto kmaj16 = [](uint32_t base, uint32_t k0) { return sdesc(base + (k0 >> 3) * 256u, 256u, 128u); };
    /* MN-major (rows = K): 8-row K groups 128 B apart, MN planes R * 16 B apart */
    auto mn128 = [](uint32_t base, uint32_t k0) { return sdesc(base + k0 * 16u, 128u, 2048u); };
    auto mn16 = [](uint32_t base, uint32_t k0) { return sdesc(base + k0 * 16u, 128u, 256u); };

    const bool backward = a.mode != MODE_FORWARD;
    for (uint32_t step = 0; step < a.nsteps && ok; ++step) {
        const uint32_t rows = a.stepRows[step], off = a.stepOff[step];
        const uint32_t tiles = (rows + kTile - 1) / kTile;
        /* weights of this step, bf16 in column planes; biases fp32 */
        for (uint32_t e = tid; e < kH * kIO; e += kThreads) {
            const uint32_t r = e / kIO, c = e % kIO;
            const float v1 = c < I ? a.p[a.oW1 + r * I + c] : 0.f;
            *reinterpret_cast<__nv_bfloat16 *>(sW1 + plane_off(kH, r, c)) = __float2bfloat16_rn(v1);
            const uint32_t o = e / kH, i = e % kH; /* W3: 16 rows (outputs) x 128 */
            const float v3 = o < O ? a.p[a.oW3 + o * kH + i] : 0.f;
            *reinterpret_cast<__nv_bfloat16 *>(sW3 + plane_off(kIO, o, i)) = __float2bfloat16_rn(v3);
        }
        for (uint32_t e = tid; e < kH * kH / 2; e += kThreads) {
            const uint32_t r = (2 * e) / kH, c = (2 * e) % kH;
            *reinterpret_cast<uint32_t *>(sW2 + plane_off(kH, r, c)) =
                pack2(a.p[a.oW2 + r * kH + c], a.p[a.oW2 + r * kH + c + 1]);
        }
        sb1[tid] = a.p[a.ob1 + tid];
        sb2[tid] = a.p[a.ob2 + tid];
        if (tid < kIO) sb3[tid] = tid < O ? a.p[a.ob3 + tid] : 0.f;
        db1[tid] = 0.f;
        db2[tid] = 0.f;
        if (tid < 32) db3[tid] = 0.f;
        float lossAcc = 0.f;
        bool first = true;
        const float invRows = 1.f / (float)rows;

        for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
            const uint32_t grow = tile * kTile + tid;
            const bool valid = grow < rows;
            const uint32_t src = valid ? (a.rowIdx ? a.rowIdx[off + grow] : off + grow) : 0u;
            {
                float xv[16];
#pragma unroll
                for (int c = 0; c < 16; ++c) xv[c] = (valid && (uint32_t)c < I) ? a.x[(size_t)src * I + c] : 0.f;
                st_row8(sX, kTile, tid, 0, xv);
                st_row8(sX, kTile, tid, 1, xv + 8);
            }
            before_mma();
            /* Z1 = X W1^T */
            if (tid == 0) {
                umma(tm + kTA, kmaj128(aX, 0), kmaj128(aW1, 0), idesc(kH, false, false), 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
            /* H1 = relu(Z1 + b1) */
            uint32_t mask1[4], mask2[4];
#pragma unroll
            for (uint32_t c16 = 0; c16 < kH / 16; ++c16) {
                float v[16];
                tmem_ld16(tm + lanes + kTA + c16 * 16, v);
                uint32_t m = 0;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float h = fmaxf(v[j] + sb1[c16 * 16 + j], 0.f);
                    m |= (h > 0.f ? 1u : 0u) << j;
                    v[j] = h;
                }
                if (c16 & 1) mask1[c16 >> 1] |= m << 16;
                else mask1[c16 >> 1] = m;
                st_row8(sH1, kTile, tid, 2 * c16, v);
                st_row8(sH1, kTile, tid, 2 * c16 + 1, v + 8);
            }
            before_mma();
            /* Z2 = H1 W2^T */
            if (tid == 0) {
                for (uint32_t k0 = 0; k0 < kH; k0 += 16)
                    umma(tm + kTB, kmaj128(aH1, k0), kmaj128(aW2, k0), idesc(kH, false, false), k0 > 0 ? 1u : 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
#pragma unroll
            for (uint32_t c16 = 0; c16 < kH / 16; ++c16) {
                float v[16];
                tmem_ld16(tm + lanes + kTB + c16 * 16, v);
                uint32_t m = 0;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float h = fmaxf(v[j] + sb2[c16 * 16 + j], 0.f);
                    m |= (h > 0.f ? 1u : 0u) << j;
                    v[j] = h;
                }
                if (c16 & 1) mask2[c16 >> 1] |= m << 16;
                else mask2[c16 >> 1] = m;
                st_row8(sH2, kTile, tid, 2 * c16, v);
                st_row8(sH2, kTile, tid, 2 * c16 + 1, v + 8);
            }
            before_mma();
            /* Y = H2 W3^T */
            if (tid == 0) {
                for (uint32_t k0 = 0; k0 < kH; k0 += 16)
                    umma(tm + kTC, kmaj128(aH2, k0), kmaj16(aW3, k0), idesc(kIO, false, false), k0 > 0 ? 1u : 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
            float y[16];
            tmem_ld16(tm + lanes + kTC, y);
#pragma unroll
            for (int o = 0; o < 16; ++o) y[o] += sb3[o];
            if (!backward) {
                if (valid)
                    for (uint32_t o = 0; o < O; ++o) a.y[(size_t)grow * O + o] = y[o];
                first = false;
                continue;
            }
            /* loss and dY = 2 w (y - t) / rows */
            float dy[16];
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                dy[o] = 0.f;
                if (valid && (uint32_t)o < O) {
                    const float d = y[o] - a.t[(size_t)src * O + o];
                    const float wo = a.w[o];
                    lossAcc += wo * d * d;
                    dy[o] = 2.f * wo * d * invRows;
                }
            }
            st_row8(sDY, kTile, tid, 0, dy);
            st_row8(sDY, kTile, tid, 1, dy + 8);
            {
                float pad[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) pad[j] = j < 16 ? dy[j] : 0.f;
                column_sums32(red, pad, db3); /* db3 holds 32 entries; 16..31 stay zero */
            }
            before_mma();
            /* dH2 = dY W3 and dW3^T (+)= H2^T dY */
            if (tid == 0) {
                umma(tm + kTA, kmaj128(aDY, 0), mn16(aW3, 0), idesc(kH, false, true), 0u);
                for (uint32_t k0 = 0; k0 < kTile; k0 += 16)
                    umma(tm + kTW3, mn128(aH2, k0), mn128(aDY, k0), idesc(kIO, true, true), (!first || k0 > 0) ? 1u : 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
            /* dZ2 = dH2 * relu'(h2), into the H2 buffer; db2 */
#pragma unroll
            for (uint32_t c32 = 0; c32 < kH / 32; ++c32) {
                float v[32];
                tmem_ld16(tm + lanes + kTA + c32 * 32, *reinterpret_cast<float(*)[16]>(v));
                tmem_ld16(tm + lanes + kTA + c32 * 32 + 16, *reinterpret_cast<float(*)[16]>(v + 16));
                const uint32_t m = mask2[c32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = ((m >> j) & 1u) ? v[j] : 0.f;
#pragma unroll
                for (int q = 0; q < 4; ++q) st_row8(sH2, kTile, tid, c32 * 4 + q, v + 8 * q);
                column_sums32(red, v, db2 + c32 * 32);
            }
            before_mma();
            /* dW2 (+)= dZ2^T H1 and dH1 = dZ2 W2 */
            if (tid == 0) {
                for (uint32_t k0 = 0; k0 < kTile; k0 += 16)
                    umma(tm + kTW2, mn128(aH2, k0), mn128(aH1, k0), idesc(kH, true, true), (!first || k0 > 0) ? 1u : 0u);
                for (uint32_t k0 = 0; k0 < kH; k0 += 16)
                    umma(tm + kTB, kmaj128(aH2, k0), mn128(aW2, k0), idesc(kH, false, true), k0 > 0 ? 1u : 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
            /* dZ1 = dH1 * relu'(h1), into the H1 buffer; db1 */
#pragma unroll
            for (uint32_t c32 = 0; c32 < kH / 32; ++c32) {
                float v[32];
                tmem_ld16(tm + lanes + kTB + c32 * 32, *reinterpret_cast<float(*)[16]>(v));
                tmem_ld16(tm + lanes + kTB + c32 * 32 + 16, *reinterpret_cast<float(*)[16]>(v + 16));
                const uint32_t m = mask1[c32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = ((m >> j) & 1u) ? v[j] : 0.f;
#pragma unroll
                for (int q = 0; q < 4; ++q) st_row8(sH1, kTile, tid, c32 * 4 + q, v + 8 * q);
                column_sums32(red, v, db1 + c32 * 32);
            }
            before_mma();
            /* dW1 (+)= dZ1^T X */
            if (tid == 0) {
                for (uint32_t k0 = 0; k0 < kTile; k0 += 16)
                    umma(tm + kTW1, mn128(aH1, k0), mn128(aX, k0), idesc(kIO, true, true), (!first || k0 > 0) ? 1u : 0u);
                umma_commit(&s_mbar);
            }
            ok = mma_wait(&s_mbar, phase, a.timeoutNs, &s_ok) && ok;
            first = false;
        }
        if (!backward) continue;

        /* this CTA's gradients and loss of the step */
        float *part = a.part + (size_t)blockIdx.x * a.nParam;
        if (first) { /* no tile in this step */
            for (uint32_t e = tid; e < a.nParam; e += kThreads) part[e] = 0.f;
        } else {
            for (uint32_t c16 = 0; c16 < kH / 16; ++c16) {
                float v[16];
                tmem_ld16(tm + lanes + kTW2 + c16 * 16, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) part[a.oW2 + tid * kH + c16 * 16 + j] = v[j];
            }
            float v[16];
            tmem_ld16(tm + lanes + kTW3, v); /* row tid = hidden unit i, columns = outputs */
            for (uint32_t o = 0; o < O; ++o) part[a.oW3 + o * kH + tid] = v[o];
            tmem_ld16(tm + lanes + kTW1, v); /* row tid = hidden unit, columns = inputs */
            for (uint32_t c = 0; c < I; ++c) part[a.oW1 + tid * I + c] = v[c];
            part[a.ob1 + tid] = db1[tid];
            part[a.ob2 + tid] = db2[tid];
            if (tid < O) part[a.ob3 + tid] = db3[tid];
        }
        for (int o = 16; o > 0; o >>= 1) lossAcc += __shfl_down_sync(0xFFFFFFFFu, lossAcc, o);
        if (lane == 0) s_loss[warp] = lossAcc;
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
        if (tid == 0) a.lossPart[blockIdx.x] = ((s_loss[0] + s_loss[1]) + s_loss[2]) + s_loss[3];
        __syncthreads();
        grid_arrive(a.bar, target, gridDim.x);
        if (!grid_wait(a.bar, target, a.timeoutNs)) {
            ok = false;
            break;
        }
        /* gradients summed over the CTAs in order; Adam */
        const uint32_t G = gridDim.x;
        for (uint32_t e = blockIdx.x * kThreads + tid; e < a.nParam; e += G * kThreads) {
            float gs = 0.f;
            for (uint32_t c = 0; c < G; ++c) gs += a.part[(size_t)c * a.nParam + e];
            if (a.mode == MODE_GRADIENTS) {
                a.g[e] = gs;
            } else {
                const float m1 = a.beta1 * a.m1[e] + (1.f - a.beta1) * gs;
                const float m2 = a.beta2 * a.m2[e] + (1.f - a.beta2) * gs * gs;
                a.m1[e] = m1;
                a.m2[e] = m2;
                a.p[e] -= a.lr * (m1 / a.c1[step]) / (sqrtf(m2 / a.c2[step]) + a.eps);
                a.g[e] = gs;
            }
        }
        if (blockIdx.x == 0 && tid == 0) {
            float l = 0.f;
            for (uint32_t c = 0; c < G; ++c) l += a.lossPart[c];
            a.losses[step] = l * invRows;
        }
        if (a.mode == MODE_TRAIN && step + 1 < a.nsteps) {
            __syncthreads();
            grid_arrive(a.bar, target, gridDim.x);
            if (!grid_wait(a.bar, target, a.timeoutNs)) {
                ok = false;
                break;
            }
        }
    }
    if (!ok && tid == 0) atomicExch(a.err, 1u);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTmemCols) : "memory");
}

/* ------------------------------------------------------------------- host */

struct CudaErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgErr : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
#define MCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) throw CudaErr(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
void malloc_n(T *&p, size_t n)
{
    p = nullptr;
    if (n) MCK(cudaMalloc((void **)&p, n * sizeof(T)));
}
template <typename T>
void free_n(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

/* parameters: W1 [H x I], b1 [H], W2 [H x H], b2 [H], W3 [O x H], b3 [O]
 * (row-major, out x in), one contiguous fp32 vector */
struct Net {
    int gpu = 0;
    uint32_t I = 0, H = 0, O = 0;
    std::string err;
    cudaStream_t stream = nullptr;
    size_t nParam = 0;
    size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
    float *d_p = nullptr, *d_g = nullptr, *d_m1 = nullptr, *d_m2 = nullptr;
    float *d_part = nullptr, *d_lossPart = nullptr;
    GridBarrier *d_bar = nullptr;
    unsigned int *d_err = nullptr;
    int maxGrid = 0;
    uint64_t adamStep = 0;
    unsigned long long timeoutNs = 2000000000ull;
    /* data buffers, grown on demand */
    float *d_x = nullptr, *d_t = nullptr, *d_w = nullptr, *d_y = nullptr, *d_losses = nullptr, *d_c = nullptr;
    uint32_t *d_idx = nullptr, *d_steps = nullptr;
    size_t capX = 0, capT = 0, capY = 0, capIdx = 0, capSteps = 0, capC = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double lastMs = 0;

    ~Net()
    {
        if (stream) cudaStreamSynchronize(stream);
        free_n(d_p); free_n(d_g); free_n(d_m1); free_n(d_m2); free_n(d_part); free_n(d_lossPart); free_n(d_bar); free_n(d_err);
        free_n(d_x); free_n(d_t); free_n(d_w); free_n(d_y); free_n(d_losses); free_n(d_c); free_n(d_idx); free_n(d_steps);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    void create(uint32_t in, uint32_t hidden, uint32_t out, uint64_t seed)
    {
        if (in == 0 || in > kIO || hidden != kH || out == 0 || out > kIO)
            throw ArgErr("the network takes 1..16 inputs, 128 hidden units and 1..16 outputs");
        I = in;
        H = hidden;
        O = out;
        oW1 = 0;
        ob1 = oW1 + (size_t)H * I;
        oW2 = ob1 + H;
        ob2 = oW2 + (size_t)H * H;
        oW3 = ob2 + H;
        ob3 = oW3 + (size_t)O * H;
        nParam = ob3 + O;
        MCK(cudaSetDevice(gpu));
        MCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        MCK(cudaEventCreate(&ev0));
        MCK(cudaEventCreate(&ev1));
        MCK(cudaFuncSetAttribute(k_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
        int sms = 0, fit = 0;
        MCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu));
        MCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_mlp, kThreads, kSmemBytes));
        if (fit < 1) throw CudaErr("the network kernel does not fit on an SM");
        maxGrid = sms; /* one CTA per SM (the shared-memory plan allows no more) */
        malloc_n(d_p, nParam);
        malloc_n(d_g, nParam);
        malloc_n(d_m1, nParam);
        malloc_n(d_m2, nParam);
        malloc_n(d_part, (size_t)maxGrid * nParam);
        malloc_n(d_lossPart, (size_t)maxGrid);
        malloc_n(d_bar, 1);
        malloc_n(d_err, 1);
        malloc_n(d_w, kIO);
        /* He initialisation (uniform, fan-in), zero biases */
        std::vector<float> p(nParam, 0.f);
        std::mt19937_64 r(seed);
        auto fill = [&](size_t off, uint32_t rows, uint32_t fan) {
            const double lim = std::sqrt(6.0 / fan);
            std::uniform_real_distribution<double> u(-lim, lim);
            for (size_t i = 0; i < (size_t)rows * fan; ++i) p[off + i] = (float)u(r);
        };
        fill(oW1, H, I);
        fill(oW2, H, H);
        fill(oW3, O, H);
        setParams(p.data(), p.size());
    }

    void setParams(const float *p, size_t n)
    {
        if (n != nParam) throw ArgErr("parameter count mismatch");
        MCK(cudaSetDevice(gpu));
        MCK(cudaMemcpyAsync(d_p, p, nParam * sizeof(float), cudaMemcpyHostToDevice, stream));
        MCK(cudaMemsetAsync(d_m1, 0, nParam * sizeof(float), stream));
        MCK(cudaMemsetAsync(d_m2, 0, nParam * sizeof(float), stream));
        adamStep = 0;
        MCK(cudaStreamSynchronize(stream));
    }

    void getParams(float *p, size_t n)
    {
        if (n != nParam) throw ArgErr("parameter count mismatch");
        MCK(cudaSetDevice(gpu));
        MCK(cudaMemcpyAsync(p, d_p, nParam * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
    }

    template <typename T>
    void grow(T *&p, size_t &cap, size_t n)
    {
        if (n <= cap) return;
        free_n(p);
        malloc_n(p, n);
        cap = n;
    }

    void upload(const float *x, const float *t, const float *w, size_t rows)
    {
        grow(d_x, capX, std::max<size_t>(rows * I, 1));
        MCK(cudaMemcpyAsync(d_x, x, rows * I * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (t) {
            grow(d_t, capT, std::max<size_t>(rows * O, 1));
            MCK(cudaMemcpyAsync(d_t, t, rows * O * sizeof(float), cudaMemcpyHostToDevice, stream));
            float wv[kIO];
            for (uint32_t o = 0; o < O; ++o) wv[o] = w ? w[o] : 1.f;
            MCK(cudaMemcpyAsync(d_w, wv, O * sizeof(float), cudaMemcpyHostToDevice, stream));
        }
    }

    /* run `nsteps` steps: step s takes stepRows[s] rows starting at entry
     * stepOff[s] of idx (or of x itself when idx is null) */
    void launch(int mode, const std::vector<uint32_t> &stepRows, const std::vector<uint32_t> &stepOff, const uint32_t *idx,
                size_t nIdx, float lr, float *losses)
    {
        const uint32_t S = (uint32_t)stepRows.size();
        uint32_t maxTiles = 1;
        for (uint32_t r : stepRows) {
            if (r == 0) throw ArgErr("empty batch");
            maxTiles = std::max(maxTiles, (r + kTile - 1) / kTile);
        }
        const int grid = (int)std::min<uint32_t>(maxTiles, (uint32_t)maxGrid);
        grow(d_steps, capSteps, 2 * (size_t)S);
        MCK(cudaMemcpyAsync(d_steps, stepRows.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        MCK(cudaMemcpyAsync(d_steps + S, stepOff.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        if (idx) {
            grow(d_idx, capIdx, nIdx);
            MCK(cudaMemcpyAsync(d_idx, idx, nIdx * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }
        /* Adam bias corrections of the steps, and the per-step losses */
        grow(d_c, capC, 3 * (size_t)S);
        std::vector<float> c(2 * (size_t)S);
        for (uint32_t s = 0; s < S; ++s) {
            const double t = (double)(adamStep + 1 + s);
            c[s] = (float)(1.0 - std::pow(0.9, t));
            c[S + s] = (float)(1.0 - std::pow(0.999, t));
        }
        MCK(cudaMemcpyAsync(d_c, c.data(), 2 * S * sizeof(float), cudaMemcpyHostToDevice, stream));
        MCK(cudaMemsetAsync(d_bar, 0, sizeof(GridBarrier), stream));
        MCK(cudaMemsetAsync(d_err, 0, sizeof(unsigned int), stream));
        Args a;
        a.I = I;
        a.O = O;
        a.nParam = (uint32_t)nParam;
        a.oW1 = (uint32_t)oW1;
        a.ob1 = (uint32_t)ob1;
        a.oW2 = (uint32_t)oW2;
        a.ob2 = (uint32_t)ob2;
        a.oW3 = (uint32_t)oW3;
        a.ob3 = (uint32_t)ob3;
        a.mode = mode;
        a.nsteps = S;
        a.stepRows = d_steps;
        a.stepOff = d_steps + S;
        a.rowIdx = idx ? d_idx : nullptr;
        a.x = d_x;
        a.t = d_t;
        a.w = d_w;
        a.y = d_y;
        a.p = d_p;
        a.m1 = d_m1;
        a.m2 = d_m2;
        a.g = d_g;
        a.part = d_part;
        a.lossPart = d_lossPart;
        a.losses = d_c + 2 * (size_t)S;
        a.c1 = d_c;
        a.c2 = d_c + S;
        a.lr = lr;
        a.beta1 = 0.9f;
        a.beta2 = 0.999f;
        a.eps = 1e-8f;
        a.bar = d_bar;
        a.timeoutNs = timeoutNs;
        a.err = d_err;
        void *args[] = {&a};
        MCK(cudaEventRecord(ev0, stream));
        if (mode == MODE_FORWARD)
            MCK(cudaLaunchKernel((const void *)k_mlp, dim3(grid), dim3(kThreads), args, kSmemBytes, stream));
        else
            MCK(cudaLaunchCooperativeKernel((const void *)k_mlp, dim3(grid), dim3(kThreads), args, kSmemBytes, stream));
        MCK(cudaEventRecord(ev1, stream));
        unsigned int e = 0;
        MCK(cudaMemcpyAsync(&e, d_err, sizeof(e), cudaMemcpyDeviceToHost, stream));
        if (losses) MCK(cudaMemcpyAsync(losses, d_c + 2 * (size_t)S, S * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
        float ms = 0;
        MCK(cudaEventElapsedTime(&ms, ev0, ev1));
        lastMs = ms;
        if (e) throw CudaErr("a wait of the network kernel timed out; its results are not valid");
        if (mode == MODE_TRAIN) adamStep += S;
    }

    void forward(const float *x, uint32_t B, float *y)
    {
        if (B == 0) return;
        MCK(cudaSetDevice(gpu));
        upload(x, nullptr, nullptr, B);
        grow(d_y, capY, (size_t)B * O);
        launch(MODE_FORWARD, {B}, {0u}, nullptr, 0, 0.f, nullptr);
        MCK(cudaMemcpyAsync(y, d_y, (size_t)B * O * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
    }

    float gradients(const float *x, const float *t, const float *w, uint32_t B, float *g, size_t n)
    {
        if (B == 0) throw ArgErr("empty batch");
        if (g && n != nParam) throw ArgErr("parameter count mismatch");
        MCK(cudaSetDevice(gpu));
        upload(x, t, w, B);
        float loss = 0.f;
        launch(MODE_GRADIENTS, {B}, {0u}, nullptr, 0, 0.f, &loss);
        if (g) {
            MCK(cudaMemcpyAsync(g, d_g, nParam * sizeof(float), cudaMemcpyDeviceToHost, stream));
            MCK(cudaStreamSynchronize(stream));
        }
        return loss;
    }

    float trainStep(const float *x, const float *t, const float *w, uint32_t B, float lr)
    {
        if (B == 0) throw ArgErr("empty batch");
        MCK(cudaSetDevice(gpu));
        upload(x, t, w, B);
        float loss = 0.f;
        launch(MODE_TRAIN, {B}, {0u}, nullptr, 0, lr, &loss);
        return loss;
    }

    /* steps over a data set: step s uses the rows idx[off_s .. off_s + rows_s) */
    void trainSteps(const float *x, const float *t, const float *w, uint32_t nRows, const uint32_t *idx, const uint32_t *rows,
                    uint32_t nsteps, float lr, float *losses)
    {
        if (nsteps == 0) return;
        if (nRows == 0 || !idx || !rows) throw ArgErr("rows and their indices are needed");
        std::vector<uint32_t> sr(rows, rows + nsteps), so(nsteps);
        size_t total = 0;
        for (uint32_t s = 0; s < nsteps; ++s) {
            so[s] = (uint32_t)total;
            total += sr[s];
        }
        for (size_t k = 0; k < total; ++k)
            if (idx[k] >= nRows) throw ArgErr("row index out of range");
        MCK(cudaSetDevice(gpu));
        upload(x, t, w, nRows);
        launch(MODE_TRAIN, sr, so, idx, total, lr, losses);
    }
};

} // namespace mlp
} // namespace bfm

struct bfm_mlp {
    bfm::mlp::Net n;
};

#define MGUARD(h, ...)                                 \
    do {                                               \
        if (!(h)) return BFM_EINVAL;                   \
        try {                                          \
            __VA_ARGS__;                               \
            return BFM_OK;                             \
        } catch (bfm::mlp::ArgErr const &ex) {         \
            (h)->n.err = ex.what();                    \
            return BFM_EINVAL;                         \
        } catch (bfm::mlp::CudaErr const &ex) {        \
            (h)->n.err = ex.what();                    \
            return BFM_ECUDA;                          \
        } catch (std::exception const &ex) {           \
            (h)->n.err = ex.what();                    \
            return BFM_ERUNTIME;                       \
        }                                              \
    } while (0)

extern "C" {

int bfm_mlp_create(int gpu, uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed, bfm_mlp **out)
{
    if (!out) return BFM_EINVAL;
    auto *h = new bfm_mlp();
    h->n.gpu = gpu;
    try {
        h->n.create(n_in, n_hidden, n_out, seed);
    } catch (bfm::mlp::ArgErr const &) {
        delete h;
        return BFM_EINVAL;
    } catch (...) {
        delete h;
        return BFM_ECUDA;
    }
    *out = h;
    return BFM_OK;
}

int bfm_mlp_destroy(bfm_mlp *h)
{
    if (!h) return BFM_EINVAL;
    delete h;
    return BFM_OK;
}

const char *bfm_mlp_last_error(const bfm_mlp *h) { return h ? h->n.err.c_str() : "null network handle"; }

int bfm_mlp_num_params(const bfm_mlp *h, size_t *n)
{
    if (!h || !n) return BFM_EINVAL;
    *n = h->n.nParam;
    return BFM_OK;
}

int bfm_mlp_set_params(bfm_mlp *h, const float *params, size_t n) { MGUARD(h, { h->n.setParams(params, n); }); }
int bfm_mlp_get_params(bfm_mlp *h, float *params, size_t n) { MGUARD(h, { h->n.getParams(params, n); }); }

int bfm_mlp_forward(bfm_mlp *h, const float *x, uint32_t batch, float *y) { MGUARD(h, { h->n.forward(x, batch, y); }); }

int bfm_mlp_gradients(bfm_mlp *h, const float *x, const float *y_target, const float *out_weight, uint32_t batch, float *grad,
                      size_t n, float *loss)
{
    MGUARD(h, {
        const float l = h->n.gradients(x, y_target, out_weight, batch, grad, n);
        if (loss) *loss = l;
    });
}

int bfm_mlp_train_step(bfm_mlp *h, const float *x, const float *y_target, const float *out_weight, uint32_t batch, float lr,
                       float *loss)
{
    MGUARD(h, {
        const float l = h->n.trainStep(x, y_target, out_weight, batch, lr);
        if (loss) *loss = l;
    });
}

int bfm_mlp_train_steps(bfm_mlp *h, const float *x, const float *y_target, const float *out_weight, uint32_t n_rows,
                        const uint32_t *row_index, const uint32_t *step_rows, uint32_t n_steps, float lr, float *losses)
{
    MGUARD(h, { h->n.trainSteps(x, y_target, out_weight, n_rows, row_index, step_rows, n_steps, lr, losses); });
}

int bfm_mlp_last_ms(const bfm_mlp *h, double *ms)
{
    if (!h || !ms) return BFM_EINVAL;
    *ms = h->n.lastMs;
    return BFM_OK;
}

} /* extern "C" */
