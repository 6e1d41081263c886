// audit.cu -- edge-degree watertight audit of a triangle mesh on the GPU.
//
// Replaces is_watertight (native/core/wtivo_core.cpp:402-464).  A closed
// 2-manifold triangle mesh has every undirected edge in exactly two faces;
// the audit reports the number of "bad edge groups": distinct undirected
// edges whose face count is not 2.
//
// The reference writes 3F 64-bit edge keys (min << 32 | max), sorts them on
// host threads and counts runs of equal keys.  Here no sort is needed: every
// edge key is counted in a device hash table (open addressing, linear
// probing, the key claimed with a 64-bit CAS, the count kept beside it),
// then one streaming pass over the table counts the keys whose count is
// not 2.  The number is the same: a run of equal keys in the sorted array is
// exactly one table entry, and its length is the entry's count.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int ATPB = 256;
constexpr unsigned long long EMPTY_KEY = ~0ull;   // no edge key: ids are < 2^31

// 64-bit mixer of SplitMix64 (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014): neighboring edge keys land
// in unrelated slots.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Counts one edge key; the probe is bounded by the table size (the table is
// at most half full, so it ends long before; a full table is reported).
__device__ __forceinline__ void count_edge(unsigned long long key, unsigned long long* keys,
                                           uint32_t* counts, unsigned long long mask, int* err)
{
    unsigned long long slot = mix64(key) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        unsigned long long k = __ldcg(keys + slot);
        if (k == EMPTY_KEY) k = atomicCAS(keys + slot, EMPTY_KEY, key);
        if (k == EMPTY_KEY || k == key) {
            atomicAdd(counts + slot, 1u);
            return;
        }
        slot = (slot + 1u) & mask;
    }
    atomicOr(err, 2);
}

// wtivo_core.cpp:420-435: the three undirected edges of every face
__global__ void __launch_bounds__(ATPB) k_edge_count(const int32_t* __restrict__ faces, uint64_t nf,
                                                     unsigned long long* keys, uint32_t* counts,
                                                     unsigned long long mask, int* err)
{
    for (uint64_t i = (uint64_t)blockIdx.x * ATPB + threadIdx.x; i < nf;
         i += (uint64_t)gridDim.x * ATPB) {
        const int32_t a = __ldg(faces + 3u * i), b = __ldg(faces + 3u * i + 1u),
                      c = __ldg(faces + 3u * i + 2u);
        if (a < 0 || b < 0 || c < 0) {   // :424 "negative vertex index"
            atomicOr(err, 1);
            continue;
        }
        const uint32_t ua = (uint32_t)a, ub = (uint32_t)b, uc = (uint32_t)c;
        count_edge(((unsigned long long)min(ua, ub) << 32) | max(ua, ub), keys, counts, mask, err);
        count_edge(((unsigned long long)min(ub, uc) << 32) | max(ub, uc), keys, counts, mask, err);
        count_edge(((unsigned long long)min(uc, ua) << 32) | max(uc, ua), keys, counts, mask, err);
    }
}

// :440-446: one bad group per distinct edge whose face count is not 2
__global__ void __launch_bounds__(ATPB) k_edge_bad(const unsigned long long* __restrict__ keys,
                                                   const uint32_t* __restrict__ counts, uint64_t cap,
                                                   unsigned long long* bad)
{
    __shared__ unsigned long long s[ATPB / 32];
    unsigned long long b = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * ATPB + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * ATPB)
        b += (keys[i] != EMPTY_KEY && counts[i] != 2u) ? 1ull : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b += __shfl_down_sync(0xffffffffu, b, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < ATPB / 32; ++w) t += s[w];
        if (t) atomicAdd(bad, t);
    }
}

}  // namespace

void edge_audit(const int32_t* d_faces, uint64_t nf, cudaStream_t s, uint64_t* bad_groups,
                uint64_t* table_bytes, uint64_t* launches)
{
    *bad_groups = 0;
    *table_bytes = 0;
    if (!nf) return;
    if (nf > (1ull << 40)) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "too many faces"};
    // capacity: a power of two at least twice the edge count (load <= 1/2)
    uint64_t cap = 1024;
    while (cap < 6u * nf) cap <<= 1;
    DevBuf<unsigned long long> keys(cap, s);
    DevBuf<uint32_t> counts(cap, s);
    DevBuf<unsigned long long> bad(1, s);
    DevBuf<int> err(1, s);
    GPUPR_CUDA(cudaMemsetAsync(keys.p, 0xFF, cap * 8u, s));
    GPUPR_CUDA(cudaMemsetAsync(counts.p, 0, cap * 4u, s));
    GPUPR_CUDA(cudaMemsetAsync(bad.p, 0, 8u, s));
    GPUPR_CUDA(cudaMemsetAsync(err.p, 0, 4u, s));
    const unsigned gf = (unsigned)std::min<uint64_t>((nf + ATPB - 1) / ATPB, (uint64_t)sm_count() * 16u);
    k_edge_count<<<gf, ATPB, 0, s>>>(d_faces, nf, keys.p, counts.p, cap - 1u, err.p);
    GPUPR_CUDA(cudaGetLastError());
    const unsigned gt = (unsigned)std::min<uint64_t>((cap + ATPB - 1) / ATPB, (uint64_t)sm_count() * 16u);
    k_edge_bad<<<gt, ATPB, 0, s>>>(keys.p, counts.p, cap, bad.p);
    GPUPR_CUDA(cudaGetLastError());
    if (launches) *launches += 2;
    unsigned long long hb = 0;
    int he = 0;
    GPUPR_CUDA(cudaMemcpyAsync(&hb, bad.p, 8u, cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaMemcpyAsync(&he, err.p, 4u, cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (he & 1) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "negative vertex index"};
    if (he) throw Error{GPUPR_ERR_INVARIANT, "edge table full"};
    *bad_groups = hb;
    *table_bytes = cap * 12u;
}

}  // namespace gpupr
