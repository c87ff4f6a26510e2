/*
 * bfm_color.cu -- species colouring of forests on the device.
 *
 * The reference colours the bond graph on the host (graphColoring,
 * graphColoring.tpp:103-439, called at UpdaterGPUScBFM_AB_Type.cu:1566-1570):
 * a depth-first walk of every component from its lowest id that gives each
 * node the smallest colour its coloured neighbours lack, then a uniform
 * rebalancing pass.  On a forest (linear chains, stars, combs) the walk
 * meets every node from exactly one coloured neighbour, its parent, so the
 * walk's colour of a node is the parity of its distance to the lowest id of
 * its component.  That parity is computed here with a parity union-find on
 * the GPU (hooking the larger root under the smaller by 64-bit CAS, pointer
 * jumping), and the host rebalancing pass of the reference runs on it, so
 * the colours are the reference's.  The union-find also yields every node's
 * component; the walk colours a component from its own nodes only, so a
 * component with a cycle (bonds >= nodes) is left to the host walk while the
 * tree components keep their device colours -- the same colours as the
 * walk over the whole graph.
 *
 * Parent words: parent id << 1 | parity of the path to that parent.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfm_color.hpp"
#include "bfm_host.hpp"

namespace bfm {
namespace {

__global__ void k_uf_init(unsigned long long *P, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) P[i] = (unsigned long long)i << 1;
}

__device__ __forceinline__ unsigned long long ld_word(const unsigned long long *p)
{
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

/* every bond (u < v) whose ends have different parents tries to hook the
 * larger parent, if it is still a root, under the smaller one, with the
 * parity that gives u and v different colours */
__global__ void k_uf_hook(const uint8_t *__restrict__ deg, const uint32_t *__restrict__ nbr, unsigned long long *P, uint32_t n,
                          unsigned int *hooks)
{
    unsigned int done = 0;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        for (uint32_t j = 0; j < deg[u]; ++j) {
            const uint32_t v = nbr[(size_t)u * 8 + j];
            if (v <= u) continue;
            const unsigned long long a = ld_word(P + u), b = ld_word(P + v);
            const uint32_t pu = (uint32_t)(a >> 1), pv = (uint32_t)(b >> 1);
            if (pu == pv) continue;
            const uint32_t big = pu > pv ? pu : pv, small = pu > pv ? pv : pu;
            const unsigned long long par = (a ^ b ^ 1ull) & 1ull;
            const unsigned long long root = (unsigned long long)big << 1;
            if (atomicCAS(P + big, root, ((unsigned long long)small << 1) | par) == root) ++done;
        }
    }
    if (done) atomicAdd(hooks, done);
}

/* pointer jumping: each node points to its grandparent, parities added */
__global__ void k_uf_jump(unsigned long long *P, uint32_t n, unsigned int *changed)
{
    unsigned int c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long a = ld_word(P + i);
        const uint32_t p = (uint32_t)(a >> 1);
        if (p == i) continue;
        const unsigned long long b = ld_word(P + p);
        const uint32_t q = (uint32_t)(b >> 1);
        if (q == p) continue;
        *reinterpret_cast<volatile unsigned long long *>(P + i) = ((unsigned long long)q << 1) | ((a ^ b) & 1ull);
        ++c;
    }
    if (c) atomicAdd(changed, c);
}

struct Dev {
    void *p[4] = {nullptr, nullptr, nullptr, nullptr};
    ~Dev()
    {
        for (void *q : p)
            if (q) cudaFree(q);
    }
};

void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace

int color_graph_device(uint32_t n, const uint8_t *deg, const uint32_t *nbr8, bool uniform, std::vector<uint32_t> &color)
{
    if (n == 0) return 0;
    Dev d;
    unsigned long long *P = nullptr;
    uint8_t *ddeg = nullptr;
    uint32_t *dnbr = nullptr;
    unsigned int *cnt = nullptr;
    ck(cudaMalloc(&d.p[0], (size_t)n * 8), "cudaMalloc");
    ck(cudaMalloc(&d.p[1], (size_t)n), "cudaMalloc");
    ck(cudaMalloc(&d.p[2], (size_t)n * 8 * sizeof(uint32_t)), "cudaMalloc");
    ck(cudaMalloc(&d.p[3], 2 * sizeof(unsigned int)), "cudaMalloc");
    P = static_cast<unsigned long long *>(d.p[0]);
    ddeg = static_cast<uint8_t *>(d.p[1]);
    dnbr = static_cast<uint32_t *>(d.p[2]);
    cnt = static_cast<unsigned int *>(d.p[3]);
    ck(cudaMemcpy(ddeg, deg, n, cudaMemcpyHostToDevice), "cudaMemcpy");
    ck(cudaMemcpy(dnbr, nbr8, (size_t)n * 8 * sizeof(uint32_t), cudaMemcpyHostToDevice), "cudaMemcpy");
    const int threads = 256;
    const int blocks = (int)std::min<uint64_t>(((uint64_t)n + threads - 1) / threads, 148ull * 32);
    k_uf_init<<<blocks, threads>>>(P, n);
    bool converged = false;
    for (int round = 0; round < 64 && !converged; ++round) {
        unsigned int hooks = 0;
        ck(cudaMemset(cnt, 0, sizeof(unsigned int)), "cudaMemset");
        k_uf_hook<<<blocks, threads>>>(ddeg, dnbr, P, n, cnt);
        ck(cudaMemcpy(&hooks, cnt, sizeof(unsigned int), cudaMemcpyDeviceToHost), "cudaMemcpy");
        bool flat = false;
        for (int jump = 0; jump < 64 && !flat; ++jump) {
            unsigned int changed = 0;
            ck(cudaMemset(cnt + 1, 0, sizeof(unsigned int)), "cudaMemset");
            k_uf_jump<<<blocks, threads>>>(P, n, cnt + 1);
            ck(cudaMemcpy(&changed, cnt + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost), "cudaMemcpy");
            flat = changed == 0;
        }
        if (!flat) return 0;
        converged = hooks == 0;
    }
    if (!converged) return 0;
    std::vector<unsigned long long> words(n);
    ck(cudaMemcpy(words.data(), P, (size_t)n * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    /* nodes and bond ends per component (indexed by its root, the lowest id) */
    std::vector<uint32_t> nodes(n, 0);
    std::vector<uint64_t> ends(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t r = (uint32_t)(words[i] >> 1);
        ++nodes[r];
        ends[r] += deg[i];
    }
    color.assign(n, kNoColor);
    bool cyclic = false;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t r = (uint32_t)(words[i] >> 1);
        if (ends[r] / 2 == (uint64_t)nodes[r] - 1) color[i] = (uint32_t)(words[i] & 1ull); /* a tree */
        else cyclic = true;
    }
    std::vector<size_t> count;
    dfs_colors_rest(n, deg, nbr8, color, count); /* components with a cycle */
    if (uniform) rebalance_colors(n, deg, nbr8, color, count);
    return cyclic ? 2 : 1;
}

} // namespace bfm
