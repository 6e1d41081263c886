// audit.cu -- edge-degree watertight audit of a triangle mesh on the GPU.
//
// Replaces is_watertight (native/core/wtivo_core.cpp:402-464).  A closed
// 2-manifold triangle mesh has every undirected edge in exactly two faces;
// the audit reports the number of "bad edge groups": distinct undirected
// edges whose face count is not 2.
//
// The reference writes 3F 64-bit edge keys (min << 32 | max), sorts them on
// host threads and counts runs of equal keys.  Here no sort is needed: every
// edge is counted in a device hash table (open addressing, linear probing),
// then one streaming pass over the table counts the edges whose count is
// not 2.  The number is the same: a run of equal keys in the sorted array is
// exactly one table entry, and its length is the entry's count.
//
// One 8-byte slot per edge: the edge as min * 2^31 + max (vertex ids are
// below 2^31, so 62 bits) and, in the top two bits, its face count
// saturating at 3 (1, 2, or "3 or more": the rule only asks whether the count
// is 2).  A slot is claimed with a 64-bit CAS that writes the edge with
// count 1 and raised with CAS; a used slot is never 0 (its count is at least
// 1), so 0 marks an empty slot.  Key and count share one 32-byte sector, so
// an edge update touches one sector of the table, not two.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int ATPB = 256;
constexpr unsigned long long EDGE_MASK = (1ull << 62) - 1ull;   // the edge's 62 bits
constexpr unsigned long long COUNT_ONE = 1ull << 62;            // count field, bits 62-63

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

// Counts one edge; the probe is bounded by the table size (the table is at
// most half full, so it ends long before; a full table is reported).
__device__ __forceinline__ void count_edge(uint32_t lo, uint32_t hi, unsigned long long* table,
                                           unsigned long long mask, int* err)
{
    const unsigned long long edge = ((unsigned long long)lo << 31) | hi;
    unsigned long long slot = mix64(edge) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        unsigned long long v = __ldcg(table + slot);
        if (v == 0ull) {
            v = atomicCAS(table + slot, 0ull, edge | COUNT_ONE);
            if (v == 0ull) return;
        }
        if ((v & EDGE_MASK) == edge) {
            // raise the count, saturating at 3 (the slot's edge never changes)
            while ((v >> 62) != 3ull) {
                const unsigned long long w = atomicCAS(table + slot, v, v + COUNT_ONE);
                if (w == v) return;
                v = w;
            }
            return;
        }
        slot = (slot + 1u) & mask;
    }
    atomicOr(err, 2);
}

// wtivo_core.cpp:420-435: the three undirected edges of every face
__global__ void __launch_bounds__(ATPB) k_edge_count(const int32_t* __restrict__ faces, uint64_t nf,
                                                     unsigned long long* table,
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
        count_edge(min(ua, ub), max(ua, ub), table, mask, err);
        count_edge(min(ub, uc), max(ub, uc), table, mask, err);
        count_edge(min(uc, ua), max(uc, ua), table, mask, err);
    }
}

// :440-446: one bad group per distinct edge whose face count is not 2
__global__ void __launch_bounds__(ATPB) k_edge_bad(const ulonglong2* __restrict__ table, uint64_t cap2,
                                                   unsigned long long* bad)
{
    __shared__ unsigned long long s[ATPB / 32];
    unsigned long long b = 0;
    // two slots per 16-byte load; a used slot holds a count of 1, 2 or 3+
    for (uint64_t i = (uint64_t)blockIdx.x * ATPB + threadIdx.x; i < cap2; i += (uint64_t)gridDim.x * ATPB) {
        const ulonglong2 v = __ldg(table + i);
        b += (v.x != 0ull && (v.x >> 62) != 2ull) ? 1ull : 0ull;
        b += (v.y != 0ull && (v.y >> 62) != 2ull) ? 1ull : 0ull;
    }
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
    DevBuf<unsigned long long> table(cap, s);
    DevBuf<unsigned long long> bad(1, s);
    DevBuf<int> err(1, s);
    GPUPR_CUDA(cudaMemsetAsync(table.p, 0, cap * 8u, s));
    GPUPR_CUDA(cudaMemsetAsync(bad.p, 0, 8u, s));
    GPUPR_CUDA(cudaMemsetAsync(err.p, 0, 4u, s));
    const unsigned gf = (unsigned)std::min<uint64_t>((nf + ATPB - 1) / ATPB, (uint64_t)sm_count() * 16u);
    k_edge_count<<<gf, ATPB, 0, s>>>(d_faces, nf, table.p, cap - 1u, err.p);
    GPUPR_CUDA(cudaGetLastError());
    const uint64_t cap2 = cap / 2u;   // cap is a power of two >= 1024
    const unsigned gt = (unsigned)std::min<uint64_t>((cap2 + ATPB - 1) / ATPB, (uint64_t)sm_count() * 16u);
    k_edge_bad<<<gt, ATPB, 0, s>>>(reinterpret_cast<const ulonglong2*>(table.p), cap2, bad.p);
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
    *table_bytes = cap * 8u;
}

}  // namespace gpupr
