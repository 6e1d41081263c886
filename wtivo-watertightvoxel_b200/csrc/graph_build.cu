// graph_build.cu -- reduced-graph build on the GPU.
//
// Replaces the host build of graph_cut_gpupr_fast_v630
// (native/gpupr/wtivo_gpupr_bindings.cpp:146-314), which streamed the full
// topology to the host in 262,144-tet chunks, built the ELL arrays with
// std::threads and uploaded them again.  Here tets/neighbors never leave HBM:
//
//   k_classify   one pass over tets: class, per-tile free counts, refs,
//                range checks                       (bindings.cpp:146-177)
//   k_tile_scan  exclusive scan of the tile counts  (serial compaction :179-187)
//   k_assign     reduced id = rank among free tets in tet order
//   k_build_rows per free tet: 4 capacities (bit-exact FP64, :65-98), ELL row,
//                reverse-slot codes, arc-pair capacity sums, t-link sums,
//                base flow (:253-291)
//
// Layout written to HBM (SoA, one 16-byte row per free node):
//   nbr int4[F], res uint4[F], rev uint8[F] (2 bits per slot),
//   pair uint4[F] (cap(v->u) + cap(u->v) per slot), term int32[F].
#include <cuda_runtime.h>
#include <stdint.h>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int TPB = 256;
constexpr int PER_THREAD = 8;
constexpr int TILE = TPB * PER_THREAD;  // tets per classification tile

// Build-phase counters/flags on the device.
struct BuildCtl {
    unsigned long long fixed_source, fixed_sink, full_refs;
    unsigned long long free_refs, terminal_edges;
    long long base_flow;
    int32_t err_range;      // neighbor index >= N
    int32_t err_build;      // invalid vertex / capacity / term range
    int32_t err_reverse;    // missing reverse slot (asymmetric adjacency)
    uint32_t err_node;
    unsigned long long free_total;
};


__device__ __forceinline__ int classify_one(int4 row, uint8_t label, uint64_t N, int* refs,
                                            int* bad)
{
    const int r[4] = {row.x, row.y, row.z, row.w};
    bool exterior = false;
    int c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (r[k] < 0) exterior = true;
        else {
            ++c;
            if ((uint64_t)(uint32_t)r[k] >= N) *bad = 1;
        }
    }
    *refs = c;
    // 0 = free, 1 = fixed source (label 0), 2 = fixed sink (hull, label != 0)
    if (label == 0) return 1;
    return exterior ? 2 : 0;
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x < 32) {
        t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : T(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;  // valid in thread 0
}

__global__ void __launch_bounds__(TPB) k_classify(uint64_t N, const int4* __restrict__ nbrs,
                                                  const uint8_t* __restrict__ labels,
                                                  uint32_t* __restrict__ tile_free,
                                                  BuildCtl* ctl)
{
    __shared__ unsigned long long sh[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    unsigned long long nfree = 0, nsrc = 0, nsnk = 0, nref = 0;
    int bad = 0;
#pragma unroll
    for (int k = 0; k < PER_THREAD; ++k) {
        const uint64_t i = base + (uint64_t)k * TPB + threadIdx.x;
        if (i < N) {
            int refs = 0;
            const int c = classify_one(__ldg(nbrs + i), __ldg(labels + i), N, &refs, &bad);
            nfree += (c == 0);
            nsrc += (c == 1);
            nsnk += (c == 2);
            nref += (unsigned long long)refs;
        }
    }
    if (bad) atomicExch(&ctl->err_range, 1);
    const unsigned long long f = block_sum(nfree, sh);
    if (threadIdx.x == 0) tile_free[blockIdx.x] = (uint32_t)f;
    const unsigned long long a = block_sum(nsrc, sh);
    if (threadIdx.x == 0 && a) atomicAdd(&ctl->fixed_source, a);
    const unsigned long long b = block_sum(nsnk, sh);
    if (threadIdx.x == 0 && b) atomicAdd(&ctl->fixed_sink, b);
    const unsigned long long r = block_sum(nref, sh);
    if (threadIdx.x == 0 && r) atomicAdd(&ctl->full_refs, r);
}

// Reduced id = rank among free tets in tet order (bindings.cpp:179-187).
__global__ void __launch_bounds__(TPB) k_assign(uint64_t N, const int4* __restrict__ nbrs,
                                                const uint8_t* __restrict__ labels,
                                                const unsigned long long* __restrict__ tile_off,
                                                int32_t* __restrict__ full_to_free,
                                                uint32_t* __restrict__ free_old)
{
    __shared__ uint32_t warp_tot[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long running = tile_off[blockIdx.x];
    for (int k = 0; k < PER_THREAD; ++k) {
        const uint64_t i = base + (uint64_t)k * TPB + threadIdx.x;
        int c = 3;  // out of range
        if (i < N) {
            int refs = 0, bad = 0;
            c = classify_one(__ldg(nbrs + i), __ldg(labels + i), N, &refs, &bad);
        }
        const unsigned m = __ballot_sync(0xffffffffu, c == 0);
        const uint32_t below = __popc(m & ((1u << lane) - 1u));
        __syncthreads();
        if (lane == 0) warp_tot[warp] = __popc(m);
        __syncthreads();
        uint32_t wbase = 0, total = 0;
#pragma unroll
        for (int w = 0; w < TPB / 32; ++w) {
            const uint32_t t = warp_tot[w];
            if (w < warp) wbase += t;
            total += t;
        }
        if (i < N) {
            if (c == 0) {
                const unsigned long long id = running + wbase + below;
                full_to_free[i] = (int32_t)id;
                free_old[id] = (uint32_t)i;
            } else {
                full_to_free[i] = (c == 1) ? -2 : -3;
            }
        }
        running += total;
    }
}

// Bit-exact restatement of capacity_exact_formula (bindings.cpp:65-98):
// IEEE double ops in the reference's order with no FMA contraction,
// correctly rounded sqrt, round-to-nearest float conversion, truncation.
// Face slot FI uses local vertices {012,013,023,123}[FI] (bindings.cpp:70);
// FI is a template argument so the vertex picks stay in registers.
template <int FI>
__device__ __forceinline__ bool face_capacity(const double (&P)[4][3], uint8_t li, uint8_t lj,
                                              double fill_T, int32_t* cap)
{
    constexpr int ia = (FI == 3) ? 1 : 0;
    constexpr int ib = (FI <= 1) ? 1 : 2;
    constexpr int ic = (FI == 0) ? 2 : 3;
    const double x1 = __dsub_rn(P[ib][0], P[ia][0]);
    const double y1 = __dsub_rn(P[ib][1], P[ia][1]);
    const double z1 = __dsub_rn(P[ib][2], P[ia][2]);
    const double x2 = __dsub_rn(P[ic][0], P[ia][0]);
    const double y2 = __dsub_rn(P[ic][1], P[ia][1]);
    const double z2 = __dsub_rn(P[ic][2], P[ia][2]);
    const double cx = __dsub_rn(__dmul_rn(y1, z2), __dmul_rn(z1, y2));
    const double cy = __dsub_rn(__dmul_rn(z1, x2), __dmul_rn(x1, z2));
    const double cz = __dsub_rn(__dmul_rn(x1, y2), __dmul_rn(y1, x2));
    const double ss = __dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz));
    const float area_f = __double2float_rn(__dmul_rn(5.0e6, __dsqrt_rn(ss)));
    const double area = (double)area_f;
    const double pen = (li != lj) ? area : __dmul_rn(area, __dadd_rn(1.0, fill_T));
    // int64 truncation then [0, 2^30): (-1, 0) -> 0 passes, NaN/inf fail.
    if (!(pen > -1.0 && pen < 1073741824.0)) return false;
    *cap = (int32_t)__double2ll_rz(pen);
    return true;
}

// Capacity of face rk of tet j in j's own direction, computed exactly as the
// thread that builds j's row computes it (same vertex order, same rounding):
// the face's three vertices go to positions 0,1,2 in the order face slot rk
// takes them, and face_capacity<0> runs the same operations on them.
__device__ __forceinline__ uint32_t reverse_capacity(const double* __restrict__ V, uint64_t nv,
                                                     int4 tj4, int rk, uint8_t lj, uint8_t li,
                                                     double fill_T)
{
    const int tj[4] = {tj4.x, tj4.y, tj4.z, tj4.w};
    const int ia = (rk == 3) ? 1 : 0;
    const int ib = (rk <= 1) ? 1 : 2;
    const int ic = (rk == 0) ? 2 : 3;
    const int pick[3] = {tj[ia], tj[ib], tj[ic]};
    double Q[4][3];
    Q[3][0] = Q[3][1] = Q[3][2] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (pick[k] < 0 || (uint64_t)pick[k] >= nv) return 0u;   // j's own row reports it
        const double* p = V + (size_t)pick[k] * 3u;
        Q[k][0] = __ldg(p);
        Q[k][1] = __ldg(p + 1);
        Q[k][2] = __ldg(p + 2);
    }
    int32_t cap = 0;
    if (!face_capacity<0>(Q, lj, li, fill_T, &cap)) return 0u;
    return (uint32_t)cap;
}

__global__ void __launch_bounds__(TPB) k_build_rows(
    uint32_t F, uint64_t N, const double* __restrict__ V, uint64_t nv,
    const int4* __restrict__ tets, const int4* __restrict__ nbrs,
    const uint8_t* __restrict__ labels, const int32_t* __restrict__ full_to_free,
    const uint32_t* __restrict__ free_old, double fill_T, int4* __restrict__ out_nbr,
    uint4* __restrict__ out_res, uint8_t* __restrict__ out_rev, uint4* __restrict__ out_pair,
    int32_t* __restrict__ out_term, uint32_t* __restrict__ out_base, BuildCtl* ctl)
{
    __shared__ unsigned long long sh[TPB / 32];
    unsigned long long refs = 0, terms = 0;
    long long base = 0;
    for (uint32_t q = blockIdx.x * TPB + threadIdx.x; q < F; q += gridDim.x * TPB) {
        const uint32_t i = __ldg(free_old + q);
        const int4 row4 = __ldg(nbrs + i);
        const int4 tet4 = __ldg(tets + i);
        const uint8_t li = __ldg(labels + i);
        const int row[4] = {row4.x, row4.y, row4.z, row4.w};
        const int tv[4] = {tet4.x, tet4.y, tet4.z, tet4.w};
        double P[4][3];
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (tv[k] < 0 || (uint64_t)tv[k] >= nv) { ok = false; P[k][0] = P[k][1] = P[k][2] = 0.0; continue; }
            const double* p = V + (size_t)tv[k] * 3u;
            P[k][0] = __ldg(p);
            P[k][1] = __ldg(p + 1);
            P[k][2] = __ldg(p + 2);
        }
        long long src = 0, snk = 0;
        int on[4] = {-1, -1, -1, -1};
        uint32_t orr[4] = {0u, 0u, 0u, 0u};
        uint32_t opr[4] = {0u, 0u, 0u, 0u};
        uint32_t rv = 0;
        int32_t caps[4];
        int32_t ms[4];
        uint8_t lj[4];
#pragma unroll
        for (int fi = 0; fi < 4; ++fi) lj[fi] = __ldg(labels + row[fi]);
        ok &= face_capacity<0>(P, li, lj[0], fill_T, &caps[0]);
        ok &= face_capacity<1>(P, li, lj[1], fill_T, &caps[1]);
        ok &= face_capacity<2>(P, li, lj[2], fill_T, &caps[2]);
        ok &= face_capacity<3>(P, li, lj[3], fill_T, &caps[3]);
#pragma unroll
        for (int fi = 0; fi < 4; ++fi) ms[fi] = __ldg(full_to_free + row[fi]);
#pragma unroll
        for (int fi = 0; fi < 4; ++fi) {
            const int j = row[fi];  // free tets have no -1 slot and j < N
            const int32_t m = ms[fi];
            const int32_t cap = caps[fi];
            if (m >= 0) {
                on[fi] = m;
                orr[fi] = (uint32_t)cap;
                ++refs;
                const int4 back = __ldg(nbrs + j);
                int rk = -1;
                if (back.w == (int)i) rk = 3;
                if (back.z == (int)i) rk = 2;
                if (back.y == (int)i) rk = 1;
                if (back.x == (int)i) rk = 0;
                if (rk < 0) {
                    atomicExch(&ctl->err_reverse, 1);
                    atomicExch(&ctl->err_node, i);
                    rk = 0;
                }
                rv |= (uint32_t)rk << (2 * fi);
                // both caps are below 2^30, so the sum fits 32 bits
                opr[fi] = (uint32_t)cap + reverse_capacity(V, nv, __ldg(tets + j), rk, lj[fi], li,
                                                           fill_T);
            } else if (m == -2) {
                src += cap;
                ++terms;
            } else {
                snk += cap;
                ++terms;
            }
        }
        const long long diff = src - snk;
        if (diff < -2147483648LL || diff > 2147483647LL) ok = false;
        if (!ok) {
            atomicExch(&ctl->err_build, 1);
            atomicExch(&ctl->err_node, i);
        }
        base += (src < snk) ? src : snk;
        if (out_base) out_base[q] = (uint32_t)((src < snk) ? src : snk);
        out_nbr[q] = make_int4(on[0], on[1], on[2], on[3]);
        out_res[q] = make_uint4(orr[0], orr[1], orr[2], orr[3]);
        out_rev[q] = (uint8_t)rv;
        out_pair[q] = make_uint4(opr[0], opr[1], opr[2], opr[3]);
        out_term[q] = (int32_t)diff;
    }
    const unsigned long long r = block_sum(refs, sh);
    if (threadIdx.x == 0 && r) atomicAdd(&ctl->free_refs, r);
    const unsigned long long t = block_sum(terms, sh);
    if (threadIdx.x == 0 && t) atomicAdd(&ctl->terminal_edges, t);
    const long long b = block_sum(base, reinterpret_cast<long long*>(sh));
    if (threadIdx.x == 0 && b) atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->base_flow), (unsigned long long)b);
}

// Reverse slots and arc-pair residual sums of a graph in the reference
// layout.  A pair sum above 2^32 - 1 (residuals the solver's uint32 arcs
// cannot hold once pushed) is reported as GPUPR_ERR_BUILD.
__global__ void __launch_bounds__(TPB) k_reverse_slots(uint32_t n, const int4* __restrict__ nbr,
                                                       const uint4* __restrict__ res,
                                                       uint8_t* __restrict__ rev,
                                                       uint4* __restrict__ pair, int32_t* err)
{
    for (uint32_t v = blockIdx.x * TPB + threadIdx.x; v < n; v += gridDim.x * TPB) {
        const int4 r4 = __ldg(nbr + v);
        const uint4 c4 = __ldg(res + v);
        const int row[4] = {r4.x, r4.y, r4.z, r4.w};
        const uint32_t own[4] = {c4.x, c4.y, c4.z, c4.w};
        uint32_t rv = 0;
        uint32_t pr[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int u = row[k];
            if (u < 0) continue;
            if ((uint32_t)u >= n) { atomicExch(err, (int)GPUPR_ERR_INVARIANT); continue; }
            const int4 b = __ldg(nbr + u);
            int rk = -1;
            if (b.w == (int)v) rk = 3;
            if (b.z == (int)v) rk = 2;
            if (b.y == (int)v) rk = 1;
            if (b.x == (int)v) rk = 0;
            if (rk < 0) { atomicExch(err, (int)GPUPR_ERR_NO_REVERSE); rk = 0; }
            rv |= (uint32_t)rk << (2 * k);
            const unsigned long long sum =
                (unsigned long long)own[k] +
                __ldg(reinterpret_cast<const uint32_t*>(res) + (size_t)u * 4u + rk);
            if (sum > 0xFFFFFFFFull) { atomicExch(err, (int)GPUPR_ERR_BUILD); continue; }
            pr[k] = (uint32_t)sum;
        }
        rev[v] = (uint8_t)rv;
        pair[v] = make_uint4(pr[0], pr[1], pr[2], pr[3]);
    }
}

__global__ void __launch_bounds__(TPB) k_scatter(uint32_t n, const uint32_t* __restrict__ free_old,
                                                 const uint32_t* __restrict__ h,
                                                 uint8_t* __restrict__ out)
{
    for (uint32_t q = blockIdx.x * TPB + threadIdx.x; q < n; q += gridDim.x * TPB)
        out[__ldg(free_old + q)] = (__ldg(h + q) != UNVIS) ? 1u : 0u;
}

__global__ void __launch_bounds__(TPB) k_partition(uint32_t n, const uint32_t* __restrict__ h,
                                                   uint8_t* __restrict__ part)
{
    for (uint32_t q = blockIdx.x * TPB + threadIdx.x; q < n; q += gridDim.x * TPB)
        part[q] = (__ldg(h + q) != UNVIS) ? 1u : 0u;
}

__global__ void __launch_bounds__(1024) k_tile_scan_generic(uint32_t ntiles,
                                                            const uint32_t* __restrict__ cnt,
                                                            unsigned long long* __restrict__ off,
                                                            unsigned long long* __restrict__ total)
{
    __shared__ unsigned long long sh[1024];
    const uint32_t per = (ntiles + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per;
    const uint32_t e = min(ntiles, b + per);
    unsigned long long s = 0;
    for (uint32_t i = b; i < e; ++i) s += cnt[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        unsigned long long v = (threadIdx.x >= (unsigned)o) ? sh[threadIdx.x - o] : 0ull;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = sh[threadIdx.x] - s;
    for (uint32_t i = b; i < e; ++i) {
        off[i] = run;
        run += cnt[i];
    }
    if (threadIdx.x == blockDim.x - 1) *total = sh[threadIdx.x];
}

int grid_for(uint64_t items, int per_block = TPB)
{
    const uint64_t want = (items + per_block - 1) / per_block;
    const uint64_t cap = (uint64_t)sm_count() * 16u;
    return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

void build_reduced_graph(const BuildInputs& in, ReducedGraph& g, BuildInfo& info,
                         cudaStream_t s, uint64_t* launches)
{
    const uint64_t N = in.N;
    const uint64_t ntiles = (N + TILE - 1) / TILE;
    DevBuf<BuildCtl> ctl(1, s);
    DevBuf<uint32_t> tile_cnt(ntiles, s);
    DevBuf<unsigned long long> tile_off(ntiles, s);
    g.full_to_free = DevBuf<int32_t>(N, s);
    GPUPR_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(BuildCtl), s));

    k_classify<<<(unsigned)ntiles, TPB, 0, s>>>(N, reinterpret_cast<const int4*>(in.d_nbrs),
                                                in.d_labels, tile_cnt.p, ctl.p);
    GPUPR_CUDA(cudaGetLastError());
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
    scan_tile_counts((uint32_t)ntiles, tile_cnt.p, tile_off.p, &ctl.p->free_total, s, launches);

    BuildCtl h{};
    GPUPR_CUDA(cudaMemcpyAsync(&h, ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    info.fixed_source = h.fixed_source;
    info.fixed_sink = h.fixed_sink;
    info.full_refs = h.full_refs;
    info.free_n = h.free_total;
    if (h.err_range) throw Error{GPUPR_ERR_NEIGHBOR_RANGE, "neighbor out of range"};
    if (h.full_refs & 1ull) throw Error{GPUPR_ERR_REFS_ODD, "neighbor reference count not even"};

    g.free_old = DevBuf<uint32_t>(info.free_n ? info.free_n : 1, s);
    k_assign<<<(unsigned)ntiles, TPB, 0, s>>>(N, reinterpret_cast<const int4*>(in.d_nbrs),
                                              in.d_labels, tile_off.p, g.full_to_free.p,
                                              g.free_old.p);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
    if (info.free_n == 0) return;
    if (info.free_n > 0x7FFFFFFFull)
        throw Error{GPUPR_ERR_TOO_MANY_NODES, ">INT32_MAX reduced nodes unsupported"};

    const uint32_t F = (uint32_t)info.free_n;
    g.n = F;
    g.nbr = DevBuf<int4>(F, s);
    g.res = DevBuf<uint32_t>((size_t)F * 4u, s);
    g.rev = DevBuf<uint8_t>(F, s);
    g.pair = DevBuf<uint32_t>((size_t)F * 4u, s);
    g.term = DevBuf<int32_t>(F, s);
    if (in.want_base_node) g.base_node = DevBuf<uint32_t>(F, s);
    k_build_rows<<<grid_for(F), TPB, 0, s>>>(
        F, N, in.d_vertices, in.nv, reinterpret_cast<const int4*>(in.d_tets),
        reinterpret_cast<const int4*>(in.d_nbrs), in.d_labels, g.full_to_free.p, g.free_old.p,
        in.fill_T, g.nbr.p, reinterpret_cast<uint4*>(g.res.p), g.rev.p,
        reinterpret_cast<uint4*>(g.pair.p), g.term.p, g.base_node.p, ctl.p);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
    GPUPR_CUDA(cudaMemcpyAsync(&h, ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (h.err_build) throw Error{GPUPR_ERR_BUILD, "invalid graph reduction/capacity state"};
    info.free_refs = h.free_refs;
    info.terminal_edges = h.terminal_edges;
    info.terminal_base_flow = h.base_flow;
    if (h.free_refs & 1ull) throw Error{GPUPR_ERR_FREE_REFS_ODD, "free reference count not even"};
    if (h.err_reverse)
        throw Error{GPUPR_ERR_NO_REVERSE,
                    "GPUPr-B200 device invariant failed: neighbor lists are not symmetric "
                    "(tet " + std::to_string(h.err_node) + ")"};
}

void scan_tile_counts(uint32_t ntiles, const uint32_t* d_cnt, unsigned long long* d_off,
                      unsigned long long* d_total, cudaStream_t s, uint64_t* launches)
{
    k_tile_scan_generic<<<1, 1024, 0, s>>>(ntiles, d_cnt, d_off, d_total);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

namespace {
void raise_reverse_error(int32_t e)
{
    if (e == GPUPR_ERR_NO_REVERSE)
        throw Error{GPUPR_ERR_NO_REVERSE,
                    "GPUPr-B200 device invariant failed: neighbor lists are not symmetric"};
    if (e == GPUPR_ERR_BUILD)
        throw Error{GPUPR_ERR_BUILD, "residual pair sum exceeds the uint32 arc range"};
    if (e) throw Error{GPUPR_ERR_INVARIANT, "GPUPr-B200 device invariant failed: neighbor id >= n"};
}
}  // namespace

void compute_reverse_slots(uint32_t n, const int4* d_nbr, const uint32_t* d_res, uint8_t* d_rev,
                           uint32_t* d_pair, cudaStream_t s, uint64_t* launches)
{
    DevBuf<int32_t> err(1, s);
    GPUPR_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t), s));
    k_reverse_slots<<<grid_for(n), TPB, 0, s>>>(n, d_nbr, reinterpret_cast<const uint4*>(d_res),
                                                d_rev, reinterpret_cast<uint4*>(d_pair), err.p);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
    int32_t e = 0;
    GPUPR_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(e), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    raise_reverse_error(e);
}

void scatter_partition(uint32_t n, const uint32_t* d_free_old, const uint32_t* d_height,
                       uint8_t* d_out, cudaStream_t s, uint64_t* launches)
{
    if (!n) return;
    k_scatter<<<grid_for(n), TPB, 0, s>>>(n, d_free_old, d_height, d_out);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

void partition_from_height(uint32_t n, const uint32_t* d_height, uint8_t* d_part, cudaStream_t s,
                           uint64_t* launches)
{
    if (!n) return;
    k_partition<<<grid_for(n), TPB, 0, s>>>(n, d_height, d_part);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
}

}  // namespace gpupr

namespace gpupr {

// Reverse slots with a caller-provided device error flag (no allocation);
// used by the allocation-free solve.
void compute_reverse_slots_noalloc(uint32_t n, const int4* d_nbr, const uint32_t* d_res,
                                   uint8_t* d_rev, uint32_t* d_pair, int32_t* d_err,
                                   cudaStream_t s)
{
    GPUPR_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int32_t), s));
    k_reverse_slots<<<grid_for(n), TPB, 0, s>>>(n, d_nbr, reinterpret_cast<const uint4*>(d_res),
                                                d_rev, reinterpret_cast<uint4*>(d_pair), d_err);
    GPUPR_CUDA(cudaGetLastError());
    int32_t e = 0;
    GPUPR_CUDA(cudaMemcpyAsync(&e, d_err, sizeof(e), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    raise_reverse_error(e);
}

}  // namespace gpupr
