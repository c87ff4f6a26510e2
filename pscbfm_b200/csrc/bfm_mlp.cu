/*
 * bfm_mlp.cu -- the small multilayer perceptron of the learned run schedule:
 * in -> hidden -> hidden -> out (ReLU), trained and evaluated on the GPU by
 * this file's own kernels.  Matrix products run on the tensor cores with
 * bf16 operands and fp32 accumulation (mma.sync m16n8k16); the master
 * parameters, biases, activations kept for the backward pass, the loss and
 * the Adam moments are fp32.
 *
 * The products are tiny (K = 16 .. 256, N <= 256, a few thousand rows), so
 * one warp computes one 16 x 8 output tile and reads its operand fragments
 * straight from global memory with arbitrary element strides; the same
 * kernel serves the forward products (X W^T), the weight gradients
 * (dH^T X) and the input gradients (dH W).
 *
 * Not in the reference: it feeds the batched ensembles' schedule
 * (per-system MCS budgets and admission order).
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pscbfm_b200.h"

namespace bfm {
namespace mlp {

/* C[m][n] (+)= sum_k A(m,k) B(k,n); A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn];
 * rows m >= M and columns n >= N are not stored, k >= K reads as zero.
 * One warp per 16 x 8 tile of C. */
__global__ void k_gemm(uint32_t M, uint32_t N, uint32_t K, const __nv_bfloat16 *__restrict__ A, uint32_t sam, uint32_t sak,
                       const __nv_bfloat16 *__restrict__ B, uint32_t sbk, uint32_t sbn, float *__restrict__ C, uint32_t ldc,
                       int accumulate, uint32_t kChunk)
{
    /* split K: blockIdx.y takes k in [y * kChunk, (y + 1) * kChunk) and
     * writes its partial tile to C + y * M * ldc (summed by k_sum_parts) */
    const uint32_t kBegin = blockIdx.y * kChunk;
    const uint32_t kEnd = kBegin + kChunk < K ? kBegin + kChunk : K;
    C += (size_t)blockIdx.y * M * ldc;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t tilesN = (N + 7) / 8;
    const uint32_t tm = warp / tilesN, tn = warp % tilesN;
    if (tm * 16 >= M) return; /* whole warp leaves together */
    const uint32_t g = lane >> 2, t = lane & 3u;
    const uint32_t m0 = tm * 16 + g, m1 = m0 + 8, n = tn * 8 + g;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (uint32_t k0 = kBegin; k0 < kEnd; k0 += 16) {
        /* A fragment: rows g and g+8, columns 2t, 2t+1 and 2t+8, 2t+9 */
        __nv_bfloat16 a[8];
        const uint32_t ks[4] = {k0 + 2 * t, k0 + 2 * t + 1, k0 + 2 * t + 8, k0 + 2 * t + 9};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k = ks[q];
            a[(q >> 1) * 4 + (q & 1)] = (m0 < M && k < kEnd) ? A[(size_t)m0 * sam + (size_t)k * sak] : zero;
            a[(q >> 1) * 4 + 2 + (q & 1)] = (m1 < M && k < kEnd) ? A[(size_t)m1 * sam + (size_t)k * sak] : zero;
        }
        /* B fragment: rows (k) 2t, 2t+1 and 2t+8, 2t+9, column g */
        __nv_bfloat16 b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k = ks[q];
            b[q] = (n < N && k < kEnd) ? B[(size_t)k * sbk + (size_t)n * sbn] : zero;
        }
        uint32_t ra[4], rb[2];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            __nv_bfloat162 p;
            p.x = a[2 * r];
            p.y = a[2 * r + 1];
            ra[r] = *reinterpret_cast<uint32_t *>(&p);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            __nv_bfloat162 p;
            p.x = b[2 * r];
            p.y = b[2 * r + 1];
            rb[r] = *reinterpret_cast<uint32_t *>(&p);
        }
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                     "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                     : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                     : "r"(ra[0]), "r"(ra[1]), "r"(ra[2]), "r"(ra[3]), "r"(rb[0]), "r"(rb[1]));
    }
    /* C fragment: rows g (c0, c1) and g+8 (c2, c3), columns 2t, 2t+1 */
    const uint32_t col = tn * 8 + 2 * t;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint32_t mm = r < 2 ? m0 : m1, nn = col + (r & 1);
        if (mm < M && nn < N) {
            float *p = C + (size_t)mm * ldc + nn;
            *p = accumulate ? *p + c[r] : c[r];
        }
    }
}

/* C = sum of the split-K partial tiles, in a fixed order (deterministic) */
__global__ void k_sum_parts(uint32_t M, uint32_t N, uint32_t ldc, uint32_t parts, const float *__restrict__ P, float *__restrict__ C)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M * N; i += gridDim.x * blockDim.x) {
        const uint32_t m = i / N, n = i % N;
        float v = 0.f;
        for (uint32_t y = 0; y < parts; ++y) v += P[(size_t)y * M * ldc + (size_t)m * ldc + n];
        C[(size_t)m * ldc + n] = v;
    }
}

/* h = relu(z + bias) (or no activation), kept in fp32 and as bf16 */
__global__ void k_bias_act(uint32_t M, uint32_t N, float *__restrict__ z, const float *__restrict__ bias, int relu,
                           __nv_bfloat16 *__restrict__ hb)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M * N; i += gridDim.x * blockDim.x) {
        float v = z[i] + bias[i % N];
        if (relu) v = fmaxf(v, 0.f);
        z[i] = v;
        if (hb) hb[i] = __float2bfloat16_rn(v);
    }
}

/* fp32 -> bf16 with zero padding of the columns n >= N (row stride ld) */
__global__ void k_to_bf16(uint32_t M, uint32_t N, uint32_t ld, const float *__restrict__ x, __nv_bfloat16 *__restrict__ xb)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M * ld; i += gridDim.x * blockDim.x) {
        const uint32_t m = i / ld, n = i % ld;
        xb[i] = __float2bfloat16_rn(n < N ? x[(size_t)m * N + n] : 0.f);
    }
}

/* loss = sum_m sum_o w_o (y - t)^2 / M; dy = 2 w_o (y - t) / M (as bf16 for
 * the products); per-block partial sums of the loss */
__global__ void k_mse(uint32_t M, uint32_t O, const float *__restrict__ y, const float *__restrict__ tgt,
                      const float *__restrict__ w, __nv_bfloat16 *__restrict__ dyb, float *__restrict__ dy, float *__restrict__ lossOut)
{
    __shared__ float part[256];
    float acc = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M * O; i += gridDim.x * blockDim.x) {
        const float d = y[i] - tgt[i];
        const float wo = w[i % O];
        acc += wo * d * d;
        const float g = 2.f * wo * d / (float)M;
        dy[i] = g;
        dyb[i] = __float2bfloat16_rn(g);
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(lossOut, part[0] / (float)M);
}

/* dz = dh * relu'(h) (h is the post-activation value), also as bf16 */
__global__ void k_relu_back(uint32_t n, const float *__restrict__ h, float *__restrict__ dh, __nv_bfloat16 *__restrict__ dhb)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = h[i] > 0.f ? dh[i] : 0.f;
        dh[i] = v;
        dhb[i] = __float2bfloat16_rn(v);
    }
}

/* db[n] = sum_m dz[m][n] */
__global__ void k_colsum(uint32_t M, uint32_t N, const float *__restrict__ dz, float *__restrict__ db)
{
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (uint32_t m = 0; m < M; ++m) s += dz[(size_t)m * N + n];
        db[n] = s;
    }
}

/* Adam (Kingma & Ba 2015) on the fp32 masters, then the bf16 copies */
__global__ void k_adam(uint32_t n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1, float *__restrict__ m2,
                       float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = b;
        p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

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

int blocks_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 8)); }

/* parameters: W1 [H x I], b1 [H], W2 [H x H], b2 [H], W3 [O x H], b3 [O]
 * (row-major, out x in), one contiguous fp32 vector */
struct Net {
    int gpu = 0;
    uint32_t I = 0, H = 0, O = 0;
    std::string err;
    cudaStream_t stream = nullptr;
    size_t nParam = 0;
    size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
    float *d_p = nullptr, *d_g = nullptr, *d_m1 = nullptr, *d_m2 = nullptr, *d_loss = nullptr;
    __nv_bfloat16 *d_pb = nullptr; /* bf16 copy of the parameters */
    uint64_t adamStep = 0;
    /* activations for the current batch capacity */
    uint32_t cap = 0;
    float *d_x = nullptr, *d_h1 = nullptr, *d_h2 = nullptr, *d_y = nullptr, *d_t = nullptr, *d_w = nullptr;
    float *d_dy = nullptr, *d_dh2 = nullptr, *d_dh1 = nullptr;
    __nv_bfloat16 *d_xb = nullptr, *d_h1b = nullptr, *d_h2b = nullptr, *d_dyb = nullptr, *d_dh2b = nullptr, *d_dh1b = nullptr;

    ~Net()
    {
        if (stream) cudaStreamSynchronize(stream);
        free_n(d_p); free_n(d_g); free_n(d_m1); free_n(d_m2); free_n(d_loss); free_n(d_pb); free_n(d_parts);
        freeActs();
        if (stream) cudaStreamDestroy(stream);
    }
    void freeActs()
    {
        free_n(d_x); free_n(d_h1); free_n(d_h2); free_n(d_y); free_n(d_t); free_n(d_w);
        free_n(d_dy); free_n(d_dh2); free_n(d_dh1);
        free_n(d_xb); free_n(d_h1b); free_n(d_h2b); free_n(d_dyb); free_n(d_dh2b); free_n(d_dh1b);
        cap = 0;
    }

    void create(uint32_t in, uint32_t hidden, uint32_t out, uint64_t seed)
    {
        if (in == 0 || in > 64 || hidden == 0 || hidden > 512 || out == 0 || out > 64)
            throw ArgErr("layer widths must be 1..64 (in, out) and 1..512 (hidden)");
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
        malloc_n(d_p, nParam);
        malloc_n(d_g, nParam);
        malloc_n(d_m1, nParam);
        malloc_n(d_m2, nParam);
        malloc_n(d_pb, nParam);
        malloc_n(d_loss, 1);
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
        refreshBf16();
        MCK(cudaStreamSynchronize(stream));
    }

    void getParams(float *p, size_t n)
    {
        if (n != nParam) throw ArgErr("parameter count mismatch");
        MCK(cudaSetDevice(gpu));
        MCK(cudaMemcpyAsync(p, d_p, nParam * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
    }

    void refreshBf16()
    {
        k_to_bf16<<<blocks_for(nParam), 256, 0, stream>>>(1, (uint32_t)nParam, (uint32_t)nParam, d_p, d_pb);
        MCK(cudaGetLastError());
    }

    void reserve(uint32_t B)
    {
        if (B <= cap) return;
        freeActs();
        malloc_n(d_x, (size_t)B * I);
        malloc_n(d_xb, (size_t)B * I);
        malloc_n(d_h1, (size_t)B * H);
        malloc_n(d_h1b, (size_t)B * H);
        malloc_n(d_h2, (size_t)B * H);
        malloc_n(d_h2b, (size_t)B * H);
        malloc_n(d_y, (size_t)B * O);
        malloc_n(d_t, (size_t)B * O);
        malloc_n(d_w, O);
        malloc_n(d_dy, (size_t)B * O);
        malloc_n(d_dyb, (size_t)B * O);
        malloc_n(d_dh2, (size_t)B * H);
        malloc_n(d_dh2b, (size_t)B * H);
        malloc_n(d_dh1, (size_t)B * H);
        malloc_n(d_dh1b, (size_t)B * H);
        cap = B;
    }

    /* split-K scratch for products with few output tiles and a long K */
    float *d_parts = nullptr;
    size_t partsCap = 0;

    void gemm(uint32_t M, uint32_t N, uint32_t K, const __nv_bfloat16 *A, uint32_t sam, uint32_t sak, const __nv_bfloat16 *B,
              uint32_t sbk, uint32_t sbn, float *C, uint32_t ldc, bool acc)
    {
        const size_t warps = (size_t)((M + 15) / 16) * ((N + 7) / 8);
        const int threads = 128;
        const int blocks = (int)((warps * 32 + threads - 1) / threads);
        /* fewer than ~1024 warps and a long K: split K into chunks of at
         * least 256, partial tiles summed in order afterwards */
        uint32_t parts = 1;
        while (!acc && warps * parts < 1024 && K / (parts * 2) >= 256) parts *= 2;
        if (parts == 1) {
            k_gemm<<<blocks, threads, 0, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, acc ? 1 : 0, K);
        } else {
            const size_t need = (size_t)parts * M * ldc;
            if (need > partsCap) {
                free_n(d_parts);
                malloc_n(d_parts, need);
                partsCap = need;
            }
            const uint32_t chunk = ((K + parts - 1) / parts + 15) / 16 * 16;
            k_gemm<<<dim3(blocks, parts), threads, 0, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, d_parts, ldc, 0, chunk);
            k_sum_parts<<<blocks_for((size_t)M * N), 256, 0, stream>>>(M, N, ldc, parts, d_parts, C);
        }
        MCK(cudaGetLastError());
    }

    /* forward pass of a batch already in d_x / d_xb */
    void forwardDevice(uint32_t B)
    {
        /* h1 = relu(x W1^T + b1) */
        gemm(B, H, I, d_xb, I, 1, d_pb + oW1, 1, I, d_h1, H, false);
        k_bias_act<<<blocks_for((size_t)B * H), 256, 0, stream>>>(B, H, d_h1, d_p + ob1, 1, d_h1b);
        gemm(B, H, H, d_h1b, H, 1, d_pb + oW2, 1, H, d_h2, H, false);
        k_bias_act<<<blocks_for((size_t)B * H), 256, 0, stream>>>(B, H, d_h2, d_p + ob2, 1, d_h2b);
        gemm(B, O, H, d_h2b, H, 1, d_pb + oW3, 1, H, d_y, O, false);
        k_bias_act<<<blocks_for((size_t)B * O), 256, 0, stream>>>(B, O, d_y, d_p + ob3, 0, nullptr);
        MCK(cudaGetLastError());
    }

    void loadInputs(const float *x, uint32_t B)
    {
        MCK(cudaMemcpyAsync(d_x, x, (size_t)B * I * sizeof(float), cudaMemcpyHostToDevice, stream));
        k_to_bf16<<<blocks_for((size_t)B * I), 256, 0, stream>>>(B, I, I, d_x, d_xb);
        MCK(cudaGetLastError());
    }

    void forward(const float *x, uint32_t B, float *y)
    {
        if (B == 0) return;
        MCK(cudaSetDevice(gpu));
        reserve(B);
        loadInputs(x, B);
        forwardDevice(B);
        MCK(cudaMemcpyAsync(y, d_y, (size_t)B * O * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
    }

    /* loss and gradients of a batch into d_g */
    float backward(const float *x, const float *t, const float *w, uint32_t B)
    {
        if (B == 0) throw ArgErr("empty batch");
        MCK(cudaSetDevice(gpu));
        reserve(B);
        loadInputs(x, B);
        MCK(cudaMemcpyAsync(d_t, t, (size_t)B * O * sizeof(float), cudaMemcpyHostToDevice, stream));
        std::vector<float> ones(O, 1.f);
        MCK(cudaMemcpyAsync(d_w, w ? w : ones.data(), O * sizeof(float), cudaMemcpyHostToDevice, stream));
        forwardDevice(B);
        MCK(cudaMemsetAsync(d_loss, 0, sizeof(float), stream));
        k_mse<<<blocks_for((size_t)B * O), 256, 0, stream>>>(B, O, d_y, d_t, d_w, d_dyb, d_dy, d_loss);
        /* layer 3: dW3 = dy^T h2, db3 = sum dy, dh2 = dy W3 */
        gemm(O, H, B, d_dyb, 1, O, d_h2b, H, 1, d_g + oW3, H, false);
        k_colsum<<<blocks_for(O), 256, 0, stream>>>(B, O, d_dy, d_g + ob3);
        gemm(B, H, O, d_dyb, O, 1, d_pb + oW3, H, 1, d_dh2, H, false);
        k_relu_back<<<blocks_for((size_t)B * H), 256, 0, stream>>>(B * H, d_h2, d_dh2, d_dh2b);
        /* layer 2 */
        gemm(H, H, B, d_dh2b, 1, H, d_h1b, H, 1, d_g + oW2, H, false);
        k_colsum<<<blocks_for(H), 256, 0, stream>>>(B, H, d_dh2, d_g + ob2);
        gemm(B, H, H, d_dh2b, H, 1, d_pb + oW2, H, 1, d_dh1, H, false);
        k_relu_back<<<blocks_for((size_t)B * H), 256, 0, stream>>>(B * H, d_h1, d_dh1, d_dh1b);
        /* layer 1 */
        gemm(H, I, B, d_dh1b, 1, H, d_xb, I, 1, d_g + oW1, I, false);
        k_colsum<<<blocks_for(H), 256, 0, stream>>>(B, H, d_dh1, d_g + ob1);
        MCK(cudaGetLastError());
        float loss = 0.f;
        MCK(cudaMemcpyAsync(&loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
        return loss;
    }

    float trainStep(const float *x, const float *t, const float *w, uint32_t B, float lr)
    {
        const float loss = backward(x, t, w, B);
        ++adamStep;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - (float)std::pow(b1, (double)adamStep), c2 = 1.f - (float)std::pow(b2, (double)adamStep);
        k_adam<<<blocks_for(nParam), 256, 0, stream>>>((uint32_t)nParam, d_p, d_g, d_m1, d_m2, lr, b1, b2, 1e-8f, c1, c2);
        refreshBf16();
        MCK(cudaStreamSynchronize(stream));
        return loss;
    }

    void gradients(float *g, size_t n)
    {
        if (n != nParam) throw ArgErr("parameter count mismatch");
        MCK(cudaMemcpyAsync(g, d_g, nParam * sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
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
        const float l = h->n.backward(x, y_target, out_weight, batch);
        h->n.gradients(grad, n);
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

} /* extern "C" */
