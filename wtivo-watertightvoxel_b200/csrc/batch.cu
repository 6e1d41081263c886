// batch.cu -- many cell graphs solved as one.
//
// Graphs of a batch are independent, so their disjoint union is one cut
// problem: pack them end to end (local vertex and neighbor ids become global
// ids), build and solve the union once, and split the results.  Compaction
// keeps tet order, so each graph's free nodes form one contiguous range and
// per-graph flows are sums over that range:
//   raw_g  = sum over free v in g of max(term_v, 0) - excess_v
//            (a preflow conserves flow per graph: what entered from the
//            source and is not left as excess went into the sink; positive
//            terminals never change during the solve)
//   base_g = sum over free v in g of min(src_v, snk_v)
#include <cuda_runtime.h>
#include <stdint.h>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int TPB = 256;

__device__ __forceinline__ uint32_t graph_of(uint64_t i, const unsigned long long* off, uint32_t G)
{
    uint32_t lo = 0, hi = G;   // largest g with off[g] <= i
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(TPB) k_batch_pack(uint64_t N, uint32_t G,
                                                    const unsigned long long* __restrict__ tet_off,
                                                    const unsigned long long* __restrict__ vert_off,
                                                    const int4* __restrict__ tets_l,
                                                    const int4* __restrict__ nbrs_l,
                                                    int4* __restrict__ tets_g, int4* __restrict__ nbrs_g)
{
    for (uint64_t i = (uint64_t)blockIdx.x * TPB + threadIdx.x; i < N; i += (uint64_t)gridDim.x * TPB) {
        const uint32_t g = graph_of(i, tet_off, G);
        const long long tb = (long long)tet_off[g], vb = (long long)vert_off[g];
        const long long ng = (long long)tet_off[g + 1] - tb;
        const long long nvg = (long long)vert_off[g + 1] - vb;
        const int4 t = __ldg(tets_l + i);
        const int4 b = __ldg(nbrs_l + i);
        // out-of-graph local ids become -2^31 (caught later as invalid vertex /
        // out-of-range neighbor) instead of aliasing into another graph
        auto vmap = [&](int x) -> int { return (x >= 0 && x < nvg) ? (int)(x + vb) : (int)0x80000000; };
        auto nmap = [&](int x) -> int {
            if (x < 0) return x;
            return x < ng ? (int)(x + tb) : 0x7FFFFFFF;
        };
        tets_g[i] = make_int4(vmap(t.x), vmap(t.y), vmap(t.z), vmap(t.w));
        nbrs_g[i] = make_int4(nmap(b.x), nmap(b.y), nmap(b.z), nmap(b.w));
    }
}

__global__ void __launch_bounds__(TPB) k_batch_free_counts(const unsigned long long* __restrict__ tet_off,
                                                           const int32_t* __restrict__ f2f,
                                                           unsigned long long* __restrict__ counts)
{
    __shared__ unsigned long long sh[TPB / 32];
    const uint32_t g = blockIdx.x;
    unsigned long long c = 0;
    for (unsigned long long i = tet_off[g] + threadIdx.x; i < tet_off[g + 1]; i += TPB)
        c += (__ldg(f2f + i) >= 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < TPB / 32; ++w) t += sh[w];
        counts[g] = t;
    }
}

__global__ void __launch_bounds__(TPB) k_batch_flows(const unsigned long long* __restrict__ free_off,
                                                     const int32_t* __restrict__ term,
                                                     const long long* __restrict__ excess,
                                                     const uint32_t* __restrict__ base_node,
                                                     long long* __restrict__ raw,
                                                     unsigned long long* __restrict__ base)
{
    __shared__ long long sr[TPB / 32];
    __shared__ unsigned long long sb[TPB / 32];
    const uint32_t g = blockIdx.x;
    long long r = 0;
    unsigned long long b = 0;
    for (unsigned long long q = free_off[g] + threadIdx.x; q < free_off[g + 1]; q += TPB) {
        const int32_t t = term[q];
        r += (t > 0 ? (long long)t : 0ll) - excess[q];
        b += base_node[q];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_down_sync(0xffffffffu, r, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = r; sb[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long tr = 0;
        unsigned long long tb = 0;
        for (int w = 0; w < TPB / 32; ++w) { tr += sr[w]; tb += sb[w]; }
        raw[g] = tr;
        base[g] = tb;
    }
}

}  // namespace

void batch_pack(uint64_t N, uint32_t G, const unsigned long long* d_tet_off,
                const unsigned long long* d_vert_off, const int32_t* d_tets_local,
                const int32_t* d_nbrs_local, int32_t* d_tets, int32_t* d_nbrs, cudaStream_t s,
                uint64_t* launches)
{
    if (!N) return;
    const uint64_t want = (N + TPB - 1) / TPB;
    const uint64_t cap = (uint64_t)sm_count() * 16u;
    k_batch_pack<<<(unsigned)(want < cap ? want : cap), TPB, 0, s>>>(
        N, G, d_tet_off, d_vert_off, reinterpret_cast<const int4*>(d_tets_local),
        reinterpret_cast<const int4*>(d_nbrs_local), reinterpret_cast<int4*>(d_tets),
        reinterpret_cast<int4*>(d_nbrs));
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

void batch_free_counts(uint32_t G, const unsigned long long* d_tet_off, const int32_t* d_full_to_free,
                       unsigned long long* d_counts, cudaStream_t s, uint64_t* launches)
{
    if (!G) return;
    k_batch_free_counts<<<G, TPB, 0, s>>>(d_tet_off, d_full_to_free, d_counts);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

void batch_flows(uint32_t G, const unsigned long long* d_free_off, const int32_t* d_term,
                 const long long* d_excess, const uint32_t* d_base_node, long long* d_raw,
                 unsigned long long* d_base, cudaStream_t s, uint64_t* launches)
{
    if (!G) return;
    k_batch_flows<<<G, TPB, 0, s>>>(d_free_off, d_term, d_excess, d_base_node, d_raw, d_base);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

}  // namespace gpupr
