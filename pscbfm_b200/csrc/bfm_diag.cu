/*
 * bfm_diag.cu -- diagnostic entry points that compare the library's device
 * arithmetic with CUDA's own libraries on the GPU (used by the tests).
 */
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdint>

#include "bfm_device.cuh"
#include "../../include/pscbfm_b200.h"

namespace {

/* out[2*k]   = the library's Philox word at (seed, subsequence, offset + k)
 * out[2*k+1] = curand() after curand_init(seed, subsequence, offset + k),
 *              the reference's use (rngs/lemonade_philox.h:48-56) */
__global__ void k_philox_vs_curand(unsigned long long seed, unsigned long long subseq, unsigned long long offset, uint32_t n,
                                   uint32_t *out)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        out[2 * k] = bfm::philox_word(seed, subseq, offset + k);
        curandStatePhilox4_32_10_t st;
        curand_init(seed, subseq, offset + k, &st);
        out[2 * k + 1] = curand(&st);
    }
}

} // namespace

extern "C" int bfm_debug_philox_vs_curand(int gpu, uint64_t seed, uint64_t subsequence, uint64_t offset, uint32_t n,
                                          uint32_t *out_pairs)
{
    if (!out_pairs || n == 0 || n > (1u << 20)) return BFM_EINVAL;
    if (cudaSetDevice(gpu) != cudaSuccess) return BFM_ECUDA;
    uint32_t *d = nullptr;
    if (cudaMalloc((void **)&d, 2 * (size_t)n * sizeof(uint32_t)) != cudaSuccess) return BFM_ECUDA;
    k_philox_vs_curand<<<(n + 255) / 256, 256>>>(seed, subsequence, offset, n, d);
    int st = BFM_OK;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(out_pairs, d, 2 * (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = BFM_ECUDA;
    cudaFree(d);
    return st;
}
