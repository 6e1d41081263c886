// labels.cu -- tet-centroid labels from a sparse unsigned distance grid.
//
// Replaces SparseUDF.sample_tet_labels (native/vdb/wtivo_vdb.cpp:1519-1584),
// the producer of the graph cut's initial labels: each tet's centroid is
// mapped into the unit query box, sampled from the narrow-band UDF with
// trilinear (box) interpolation, and labelled 0 (inside the band: source)
// when the sample is at most the threshold, else 1.  The reference runs this
// on host threads against an OpenVDB tree; here one GPU thread per tet reads
// a brick grid (8^3-voxel bricks behind a dense brick table) kept in HBM, so
// the labels are produced where the cut consumes them.
//
// Arithmetic follows the reference step by step in IEEE double (no FMA
// contraction: explicit __d*_rn operations), the index transform of an
// OpenVDB linear transform (world * (1 / voxel_size)), and OpenVDB 12.0.1's
// BoxSampler (openvdb/tools/Interpolation.h): the 8 voxels around
// floor(index), lerped along z, then y, then x, each lerp a + float((b-a)*w)
// with float values and a double weight.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr int LTPB = 256;

struct GridView {
    double inv_h;
    int32_t origin[3];
    int32_t dims[3];
    float background;
    const int32_t* __restrict__ table;
    const float* __restrict__ values;
};

__device__ __forceinline__ float voxel(const GridView& g, long long i, long long j, long long k)
{
    i -= g.origin[0];
    j -= g.origin[1];
    k -= g.origin[2];
    if (i < 0 || j < 0 || k < 0) return g.background;
    const long long bx = i >> 3, by = j >> 3, bz = k >> 3;
    if (bx >= g.dims[0] || by >= g.dims[1] || bz >= g.dims[2]) return g.background;
    const int32_t b = __ldg(g.table + (bx * g.dims[1] + by) * g.dims[2] + bz);
    if (b < 0) return g.background;
    return __ldg(g.values + (size_t)b * 512u + (size_t)(((i & 7) * 8 + (j & 7)) * 8 + (k & 7)));
}

// one lerp of the box sampler: a + float((b - a) * w)
__device__ __forceinline__ float box_lerp(float a, float b, double w)
{
    const float diff = __fsub_rn(b, a);
    return __fadd_rn(a, __double2float_rn(__dmul_rn((double)diff, w)));
}

// floor of an index coordinate, clamped far outside any grid
__device__ __forceinline__ long long floor_index(double x, double& f)
{
    f = floor(x);
    const double lim = 1099511627776.0;   // 2^40 voxels
    return (long long)fmin(fmax(f, -lim), lim);
}

__global__ void __launch_bounds__(LTPB) k_sample_labels(GridView g, const double* __restrict__ V,
                                                        uint64_t nv, const int4* __restrict__ tets,
                                                        uint64_t nt, double3 bmin, double3 span,
                                                        double scale, double padding,
                                                        double threshold, uint8_t* labels,
                                                        float* udf, int* err)
{
    for (uint64_t i = (uint64_t)blockIdx.x * LTPB + threadIdx.x; i < nt; i += (uint64_t)gridDim.x * LTPB) {
        const int4 t = __ldg(tets + i);
        const int q[4] = {t.x, t.y, t.z, t.w};
        double cx = 0.0, cy = 0.0, cz = 0.0;
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {   // wtivo_vdb.cpp:1563-1570
            if (q[k] < 0 || (uint64_t)q[k] >= nv) {
                ok = false;
                break;
            }
            const double* p = V + 3u * (uint64_t)q[k];
            cx = __dadd_rn(cx, __ldg(p));
            cy = __dadd_rn(cy, __ldg(p + 1));
            cz = __dadd_rn(cz, __ldg(p + 2));
        }
        if (!ok) {
            atomicOr(err, 1);
            continue;
        }
        cx = __dmul_rn(cx, 0.25);
        cy = __dmul_rn(cy, 0.25);
        cz = __dmul_rn(cz, 0.25);
        // :1572-1574, then the grid's index transform
        const double nx = __dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn(cx, bmin.x), span.x), scale), padding);
        const double ny = __dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn(cy, bmin.y), span.y), scale), padding);
        const double nz = __dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn(cz, bmin.z), span.z), scale), padding);
        const double x = __dmul_rn(nx, g.inv_h), y = __dmul_rn(ny, g.inv_h), z = __dmul_rn(nz, g.inv_h);
        double fx, fy, fz;
        const long long ix = floor_index(x, fx), iy = floor_index(y, fy), iz = floor_index(z, fz);
        const double u = __dsub_rn(x, fx), v = __dsub_rn(y, fy), w = __dsub_rn(z, fz);
        const float d000 = voxel(g, ix, iy, iz), d001 = voxel(g, ix, iy, iz + 1);
        const float d010 = voxel(g, ix, iy + 1, iz), d011 = voxel(g, ix, iy + 1, iz + 1);
        const float d100 = voxel(g, ix + 1, iy, iz), d101 = voxel(g, ix + 1, iy, iz + 1);
        const float d110 = voxel(g, ix + 1, iy + 1, iz), d111 = voxel(g, ix + 1, iy + 1, iz + 1);
        const float val = box_lerp(box_lerp(box_lerp(d000, d001, w), box_lerp(d010, d011, w), v),
                                   box_lerp(box_lerp(d100, d101, w), box_lerp(d110, d111, w), v), u);
        labels[i] = ((double)val <= threshold) ? 0u : 1u;   // :1576
        if (udf) udf[i] = val;
    }
}

}  // namespace

void sample_tet_labels(const BrickGridDesc& grid, const double* d_vertices, uint64_t nv,
                       const int32_t* d_tets, uint64_t nt, const double* bmin, const double* bmax,
                       double padding, double threshold, uint8_t* d_labels, float* d_udf,
                       cudaStream_t s, uint64_t* launches)
{
    const double sx = bmax[0] - bmin[0], sy = bmax[1] - bmin[1], sz = bmax[2] - bmin[2];
    if (!(sx > 0 && sy > 0 && sz > 0))   // :1546-1547
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "SparseUDF.sample_tet_labels: degenerate bbox"};
    if (!nt) return;
    GridView g;
    g.inv_h = 1.0 / grid.voxel_size;
    for (int k = 0; k < 3; ++k) {
        g.origin[k] = grid.origin[k];
        g.dims[k] = grid.dims[k];
    }
    g.background = grid.background;
    g.table = grid.d_table;
    g.values = grid.d_values;
    DevBuf<int> err(1, s);
    GPUPR_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    const unsigned blocks = (unsigned)std::min<uint64_t>((nt + LTPB - 1) / LTPB, (uint64_t)sm_count() * 16u);
    k_sample_labels<<<blocks, LTPB, 0, s>>>(g, d_vertices, nv, reinterpret_cast<const int4*>(d_tets), nt,
                                            make_double3(bmin[0], bmin[1], bmin[2]),
                                            make_double3(sx, sy, sz), 1.0 - 2.0 * padding, padding,
                                            threshold, d_labels, d_udf, err.p);
    GPUPR_CUDA(cudaGetLastError());
    if (launches) *launches += 1;
    int he = 0;
    GPUPR_CUDA(cudaMemcpyAsync(&he, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (he) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "SparseUDF.sample_tet_labels: tet index out of range"};
}

}  // namespace gpupr
