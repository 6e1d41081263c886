// surface.cu -- cut-surface extraction on the GPU.
//
// Replaces surface_extraction_topology_cuda
// (native/gpupr/wtivo_gpupr_bindings.cpp:400-577), which streamed the full
// topology to the host twice.  Same output, computed where the topology
// lives:
//
//   k_surf_count   faces per 2048-tet tile: every slot of a label-0 tet whose
//                  neighbor is -1 or has a label != 0 (:446-454, :486-490)
//   scan           tile offsets (the reference's chunk/thread offsets :462-463,
//                  :495-497: contiguous ranges concatenated in order, i.e.
//                  plain tet order, then slot order)
//   k_surf_emit    sorted face vertices and orientation by the sign of the
//                  opposite-vertex volume, bit-exact FP64 (:511-536); marks
//                  used vertices
//   k_used_*       compact used vertices in original order (:543-546)
//   k_surf_remap   faces in compacted ids + vertex gather (:548-569)
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <memory>
#include <string>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int TPB = 256;
constexpr int PER = 8;
constexpr int TILE = TPB * PER;

struct SurfCtl {
    int32_t err_range;
    int32_t err_vertex;
    unsigned long long faces;
    unsigned long long used;
};

__constant__ int c_flut[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
__constant__ int c_opp[4] = {3, 2, 1, 0};

__device__ __forceinline__ int tet_faces(uint64_t i, uint64_t N, const int4* nbrs,
                                         const uint8_t* lp, int* bad, uint32_t* mask)
{
    *mask = 0;
    if (i >= N || __ldg(lp + i) != 0u) return 0;
    const int4 r4 = __ldg(nbrs + i);
    const int r[4] = {r4.x, r4.y, r4.z, r4.w};
    int c = 0;
#pragma unroll
    for (int fi = 0; fi < 4; ++fi) {
        const int j = r[fi];
        bool take;
        if (j < 0) take = true;
        else if ((uint64_t)(uint32_t)j >= N) { *bad = 1; take = false; }
        else take = __ldg(lp + j) != 0u;
        if (take) { ++c; *mask |= 1u << fi; }
    }
    return c;
}

__global__ void __launch_bounds__(TPB) k_surf_count(uint64_t N, const int4* __restrict__ nbrs,
                                                    const uint8_t* __restrict__ lp,
                                                    uint32_t* __restrict__ tile_cnt, SurfCtl* ctl)
{
    __shared__ uint32_t sh[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    uint32_t c = 0;
    int bad = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        uint32_t m;
        c += tet_faces(base + (uint64_t)k * TPB + threadIdx.x, N, nbrs, lp, &bad, &m);
    }
    if (bad) atomicExch(&ctl->err_range, 1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < TPB / 32; ++w) t += sh[w];
        tile_cnt[blockIdx.x] = t;
    }
}

// Exclusive scan of small per-thread counts across the block, in thread order.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t c, uint32_t* wtot, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    uint32_t wb = 0, t = 0;
#pragma unroll
    for (int w = 0; w < TPB / 32; ++w) {
        const uint32_t v = wtot[w];
        if (w < warp) wb += v;
        t += v;
    }
    *total = t;
    return wb + x - c;
}

__global__ void __launch_bounds__(TPB) k_surf_emit(uint64_t N, const int4* __restrict__ tets,
                                                   const int4* __restrict__ nbrs,
                                                   const uint8_t* __restrict__ lp,
                                                   const double* __restrict__ V, uint64_t nv,
                                                   const unsigned long long* __restrict__ tile_off,
                                                   int3* __restrict__ raw, uint8_t* __restrict__ used,
                                                   SurfCtl* ctl)
{
    __shared__ uint32_t wtot[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    unsigned long long running = tile_off[blockIdx.x];
    for (int k = 0; k < PER; ++k) {
        const uint64_t i = base + (uint64_t)k * TPB + threadIdx.x;
        int bad = 0;
        uint32_t mask = 0;
        const uint32_t c = tet_faces(i, N, nbrs, lp, &bad, &mask);
        uint32_t total = 0;
        const uint32_t ex = block_excl_scan(c, wtot, &total);
        if (c) {
            unsigned long long pos = running + ex;
            const int4 t4 = __ldg(tets + i);
            const int tr[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
            for (int fi = 0; fi < 4; ++fi) {
                if (!(mask & (1u << fi))) continue;
                int a0 = tr[c_flut[fi][0]], b0 = tr[c_flut[fi][1]], c0 = tr[c_flut[fi][2]];
                const int fourth = tr[c_opp[fi]];
                if (a0 < 0 || b0 < 0 || c0 < 0 || fourth < 0 || (uint64_t)a0 >= nv ||
                    (uint64_t)b0 >= nv || (uint64_t)c0 >= nv || (uint64_t)fourth >= nv) {
                    atomicExch(&ctl->err_vertex, 1);
                    raw[pos++] = make_int3(0, 0, 0);
                    continue;
                }
                int t;
                if (a0 > b0) { t = a0; a0 = b0; b0 = t; }
                if (b0 > c0) { t = b0; b0 = c0; c0 = t; }
                if (a0 > b0) { t = a0; a0 = b0; b0 = t; }
                const double* v0 = V + (size_t)a0 * 3u;
                const double* v1 = V + (size_t)b0 * 3u;
                const double* v2 = V + (size_t)c0 * 3u;
                const double* vp = V + (size_t)fourth * 3u;
                const double x1 = __dsub_rn(v1[0], v0[0]), y1 = __dsub_rn(v1[1], v0[1]), z1 = __dsub_rn(v1[2], v0[2]);
                const double x2 = __dsub_rn(v2[0], v0[0]), y2 = __dsub_rn(v2[1], v0[1]), z2 = __dsub_rn(v2[2], v0[2]);
                const double cx = __dsub_rn(__dmul_rn(y1, z2), __dmul_rn(z1, y2));
                const double cy = __dsub_rn(__dmul_rn(z1, x2), __dmul_rn(x1, z2));
                const double cz = __dsub_rn(__dmul_rn(x1, y2), __dmul_rn(y1, x2));
                const double px = __dsub_rn(vp[0], v0[0]), py = __dsub_rn(vp[1], v0[1]), pz = __dsub_rn(vp[2], v0[2]);
                const double vol = __dadd_rn(__dadd_rn(__dmul_rn(cx, px), __dmul_rn(cy, py)), __dmul_rn(cz, pz));
                const bool neg = vol < 0.0;
                raw[pos++] = make_int3(a0, neg ? b0 : c0, neg ? c0 : b0);
                used[a0] = 1u;
                used[b0] = 1u;
                used[c0] = 1u;
            }
        }
        if (bad) atomicExch(&ctl->err_range, 1);
        running += total;
    }
}

__global__ void __launch_bounds__(TPB) k_used_count(uint64_t nv, const uint8_t* __restrict__ used,
                                                    uint32_t* __restrict__ tile_cnt)
{
    __shared__ uint32_t sh[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const uint64_t i = base + (uint64_t)k * TPB + threadIdx.x;
        if (i < nv) c += used[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < TPB / 32; ++w) t += sh[w];
        tile_cnt[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(TPB) k_used_assign(uint64_t nv, const uint8_t* __restrict__ used,
                                                     const unsigned long long* __restrict__ tile_off,
                                                     int32_t* __restrict__ remap)
{
    __shared__ uint32_t wtot[TPB / 32];
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    unsigned long long running = tile_off[blockIdx.x];
    for (int k = 0; k < PER; ++k) {
        const uint64_t i = base + (uint64_t)k * TPB + threadIdx.x;
        const uint32_t c = (i < nv) ? used[i] : 0u;
        uint32_t total = 0;
        const uint32_t ex = block_excl_scan(c, wtot, &total);
        if (i < nv) remap[i] = c ? (int32_t)(running + ex) : -1;
        running += total;
    }
}

__global__ void __launch_bounds__(TPB) k_surf_remap(uint64_t F, const int3* __restrict__ raw,
                                                    const int32_t* __restrict__ remap,
                                                    int3* __restrict__ faces)
{
    for (uint64_t f = (uint64_t)blockIdx.x * TPB + threadIdx.x; f < F; f += (uint64_t)gridDim.x * TPB) {
        const int3 r = raw[f];
        faces[f] = make_int3(__ldg(remap + r.x), __ldg(remap + r.y), __ldg(remap + r.z));
    }
}

__global__ void __launch_bounds__(TPB) k_vert_gather(uint64_t nv, const int32_t* __restrict__ remap,
                                                     const double* __restrict__ V,
                                                     double* __restrict__ out)
{
    for (uint64_t i = (uint64_t)blockIdx.x * TPB + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * TPB) {
        const int32_t r = remap[i];
        if (r < 0) continue;
        out[(size_t)r * 3u] = V[i * 3u];
        out[(size_t)r * 3u + 1u] = V[i * 3u + 1u];
        out[(size_t)r * 3u + 2u] = V[i * 3u + 2u];
    }
}

// Result of the last gpupr_surface_count on this thread.
struct SurfState {
    int device = -1;
    cudaStream_t stream = nullptr;
    uint64_t faces = 0, used = 0, nv = 0;
    DevBuf<int3> raw;
    DevBuf<int32_t> remap;
    DevBuf<double> vcopy;      // device copy of host vertices
    const double* d_vertices = nullptr;
};
thread_local std::unique_ptr<SurfState> t_surf;

int grid_for(uint64_t items)
{
    const uint64_t want = (items + TPB - 1) / TPB;
    const uint64_t cap = (uint64_t)sm_count() * 16u;
    return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

void surface_count(const uint8_t* labels, int l_dev, const double* vertices, uint64_t nv, int v_dev,
                   const int32_t* d_tets, const int32_t* d_nbrs, uint64_t N, uint64_t* n_faces,
                   uint64_t* n_used, cudaStream_t s)
{
    t_surf.reset();
    auto st = std::make_unique<SurfState>();
    GPUPR_CUDA(cudaGetDevice(&st->device));
    st->stream = s;
    st->nv = nv;
    DevBuf<uint8_t> dlab;
    const uint8_t* d_labels = labels;
    if (!l_dev && N) {
        dlab = DevBuf<uint8_t>(N, s);
        host_to_device(dlab.p, labels, N, s);
        d_labels = dlab.p;
    }
    st->d_vertices = vertices;
    if (!v_dev && nv) {
        st->vcopy = DevBuf<double>(nv * 3u, s);
        host_to_device(st->vcopy.p, vertices, nv * 24u, s);
        st->d_vertices = st->vcopy.p;
    }
    uint64_t launches = 0;
    const uint64_t nt = (N + TILE - 1) / TILE;
    DevBuf<SurfCtl> ctl(1, s);
    GPUPR_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(SurfCtl), s));
    SurfCtl h{};
    if (N) {
        DevBuf<uint32_t> cnt(nt, s);
        DevBuf<unsigned long long> off(nt, s);
        k_surf_count<<<(unsigned)nt, TPB, 0, s>>>(N, reinterpret_cast<const int4*>(d_nbrs), d_labels,
                                                  cnt.p, ctl.p);
        GPUPR_CUDA(cudaGetLastError());
        scan_tile_counts((uint32_t)nt, cnt.p, off.p, &ctl.p->faces, s, &launches);
        GPUPR_CUDA(cudaMemcpyAsync(&h, ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        GPUPR_CUDA(cudaStreamSynchronize(s));
        if (h.err_range) throw Error{GPUPR_ERR_NEIGHBOR_RANGE, "surface neighbor out of range"};
        st->faces = h.faces;
        DevBuf<uint8_t> used(nv ? nv : 1, s);
        GPUPR_CUDA(cudaMemsetAsync(used.p, 0, nv ? nv : 1, s));
        st->raw = DevBuf<int3>(st->faces ? st->faces : 1, s);
        k_surf_emit<<<(unsigned)nt, TPB, 0, s>>>(N, reinterpret_cast<const int4*>(d_tets),
                                                 reinterpret_cast<const int4*>(d_nbrs), d_labels,
                                                 st->d_vertices, nv, off.p, st->raw.p, used.p, ctl.p);
        GPUPR_CUDA(cudaGetLastError());
        const uint64_t vt = (nv + TILE - 1) / TILE;
        if (nv) {
            DevBuf<uint32_t> vcnt(vt, s);
            DevBuf<unsigned long long> voff(vt, s);
            k_used_count<<<(unsigned)vt, TPB, 0, s>>>(nv, used.p, vcnt.p);
            GPUPR_CUDA(cudaGetLastError());
            scan_tile_counts((uint32_t)vt, vcnt.p, voff.p, &ctl.p->used, s, &launches);
            st->remap = DevBuf<int32_t>(nv, s);
            k_used_assign<<<(unsigned)vt, TPB, 0, s>>>(nv, used.p, voff.p, st->remap.p);
            GPUPR_CUDA(cudaGetLastError());
        }
        GPUPR_CUDA(cudaMemcpyAsync(&h, ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        GPUPR_CUDA(cudaStreamSynchronize(s));
        if (h.err_vertex) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "surface invalid tet vertex index"};
        st->used = h.used;
    }
    *n_faces = st->faces;
    *n_used = st->used;
    t_surf = std::move(st);
}

void surface_fetch(int32_t* faces, double* verts, int out_dev, cudaStream_t s)
{
    if (!t_surf) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "gpupr_surface_fetch without a prior count"};
    SurfState& st = *t_surf;
    GPUPR_CUDA(cudaSetDevice(st.device));
    if (st.faces) {
        int3* dfaces = reinterpret_cast<int3*>(faces);
        DevBuf<int3> tmpf;
        if (!out_dev) { tmpf = DevBuf<int3>(st.faces, s); dfaces = tmpf.p; }
        k_surf_remap<<<grid_for(st.faces), TPB, 0, s>>>(st.faces, st.raw.p, st.remap.p, dfaces);
        GPUPR_CUDA(cudaGetLastError());
        if (!out_dev) device_to_host(faces, dfaces, st.faces * 12u, s);
        double* dverts = verts;
        DevBuf<double> tmpv;
        if (!out_dev) { tmpv = DevBuf<double>(st.used * 3u, s); dverts = tmpv.p; }
        k_vert_gather<<<grid_for(st.nv), TPB, 0, s>>>(st.nv, st.remap.p, st.d_vertices, dverts);
        GPUPR_CUDA(cudaGetLastError());
        if (!out_dev) device_to_host(verts, dverts, st.used * 24u, s);
        GPUPR_CUDA(cudaStreamSynchronize(s));
    }
    t_surf.reset();
}

}  // namespace gpupr
