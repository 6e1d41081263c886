/*
 * synth.c -- seeded synthetic inputs for the graph-cut path.
 *
 * The reference produces its cell graph with CGAL (Delaunay of a point
 * proxy, native/core/wtivo_core.cpp:72-165) and its tet labels with an
 * OpenVDB unsigned-distance field sampled at tet centroids
 * (native/vdb/wtivo_vdb.cpp:1519-1584).  Neither library exists here, so
 * these host routines stand in for them:
 *
 *  - synth_lattice: a jittered Kuhn (Freudenthal) tetrahedralization of a
 *    box, 6 tets per cube, with neighbors computed analytically in the
 *    reference's CelloCut slot convention (slot fi shares face
 *    {012,013,023,123}[fi], i.e. the tet opposite local vertex 3-fi;
 *    -1 on the hull).  Cubes are emitted in Morton order so that tet ids are
 *    spatially coherent, as CGAL's spatially sorted insertion makes them.
 *  - synth_udf_labels: label 0 iff the exact point-to-triangle distance from
 *    a tet centroid (mean of its 4 vertices, as wtivo_vdb.cpp:1561-1570) to
 *    the mesh is <= threshold, else 1 (wtivo_vdb.cpp:1577-1578).  Centroids
 *    and mesh may be given separate affine maps so the reference's label
 *    query coordinates can be mimicked.
 *
 * Everything is deterministic for a given seed (hash-based jitter) and
 * independent of the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

/* permutations of the axes; tet p of a cube walks e[P[p][0]], e[P[p][1]],
 * e[P[p][2]] from the cube's low corner to its high corner. */
static const int PERM[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

static int perm_index(int a, int b, int c)
{
    for (int p = 0; p < 6; ++p)
        if (PERM[p][0] == a && PERM[p][1] == b && PERM[p][2] == c) return p;
    return -1;
}

static inline uint64_t spread3(uint64_t v)
{
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

static inline uint32_t compact3(uint64_t v)
{
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v ^ (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v ^ (v >> 8)) & 0x1F0000FF0000FFull;
    v = (v ^ (v >> 16)) & 0x1F00000000FFFFull;
    v = (v ^ (v >> 32)) & 0x1FFFFFull;
    return (uint32_t)v;
}

/* Returns the number of tets (6*nx*ny*nz) or -1 on bad arguments.
 * V[(nx+1)(ny+1)(nz+1)*3], tets/nbrs[6*nx*ny*nz*4],
 * cube_rank scratch[nx*ny*nz]. jitter is a fraction of the cell size. */
int64_t synth_lattice(int nx, int ny, int nz, const double* lo, const double* h,
                      double jitter, uint64_t seed, double* V, int32_t* tets,
                      int32_t* nbrs, int32_t* cube_rank)
{
    if (nx < 1 || ny < 1 || nz < 1) return -1;
    const int64_t ncube = (int64_t)nx * ny * nz;
    if (ncube * 6 > 0x7FFFFFFFll) return -1;
    const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1;

#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < vz; ++z)
        for (int64_t y = 0; y < vy; ++y)
            for (int64_t x = 0; x < vx; ++x) {
                const int64_t id = x + vx * (y + vy * z);
                const uint64_t hs = mix64(seed ^ mix64((uint64_t)id));
                double j[3];
                j[0] = (u01(hs) - 0.5) * 2.0 * jitter;
                j[1] = (u01(mix64(hs + 1)) - 0.5) * 2.0 * jitter;
                j[2] = (u01(mix64(hs + 2)) - 0.5) * 2.0 * jitter;
                /* boundary vertices stay on the box faces */
                if (x == 0 || x == vx - 1) j[0] = 0.0;
                if (y == 0 || y == vy - 1) j[1] = 0.0;
                if (z == 0 || z == vz - 1) j[2] = 0.0;
                V[id * 3 + 0] = lo[0] + ((double)x + j[0]) * h[0];
                V[id * 3 + 1] = lo[1] + ((double)y + j[1]) * h[1];
                V[id * 3 + 2] = lo[2] + ((double)z + j[2]) * h[2];
            }

    /* Morton ranks of the cubes */
    int bits = 0;
    while ((1 << bits) < nx || (1 << bits) < ny || (1 << bits) < nz) ++bits;
    const uint64_t codes = 1ull << (3 * bits);
    int64_t rank = 0;
    for (uint64_t m = 0; m < codes; ++m) {
        const uint32_t x = compact3(m), y = compact3(m >> 1), z = compact3(m >> 2);
        if ((int)x >= nx || (int)y >= ny || (int)z >= nz) continue;
        cube_rank[x + (int64_t)nx * (y + (int64_t)ny * z)] = (int32_t)rank++;
    }

#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t c = x + nx * (y + ny * z);
                const int64_t r = cube_rank[c];
                for (int p = 0; p < 6; ++p) {
                    const int64_t t = r * 6 + p;
                    int64_t cur[3] = {x, y, z};
                    int32_t vid[4];
                    for (int k = 0; k < 4; ++k) {
                        if (k > 0) cur[PERM[p][k - 1]] += 1;
                        vid[k] = (int32_t)(cur[0] + vx * (cur[1] + vy * cur[2]));
                    }
                    for (int k = 0; k < 4; ++k) tets[t * 4 + k] = vid[k];
                    const int a = PERM[p][0], b = PERM[p][1], cc = PERM[p][2];
                    /* slot 0: face opposite v3 -> cube - e_c, perm (c,a,b) */
                    {
                        int64_t q[3] = {x, y, z};
                        q[cc] -= 1;
                        int32_t nb = -1;
                        if (q[0] >= 0 && q[1] >= 0 && q[2] >= 0) {
                            const int64_t qc = q[0] + nx * (q[1] + ny * q[2]);
                            nb = (int32_t)((int64_t)cube_rank[qc] * 6 + perm_index(cc, a, b));
                        }
                        nbrs[t * 4 + 0] = nb;
                    }
                    /* slot 1: face opposite v2 -> same cube, perm (a,c,b) */
                    nbrs[t * 4 + 1] = (int32_t)(r * 6 + perm_index(a, cc, b));
                    /* slot 2: face opposite v1 -> same cube, perm (b,a,c) */
                    nbrs[t * 4 + 2] = (int32_t)(r * 6 + perm_index(b, a, cc));
                    /* slot 3: face opposite v0 -> cube + e_a, perm (b,c,a) */
                    {
                        int64_t q[3] = {x, y, z};
                        q[a] += 1;
                        int32_t nb = -1;
                        if (q[0] < nx && q[1] < ny && q[2] < nz) {
                            const int64_t qc = q[0] + nx * (q[1] + ny * q[2]);
                            nb = (int32_t)((int64_t)cube_rank[qc] * 6 + perm_index(b, cc, a));
                        }
                        nbrs[t * 4 + 3] = nb;
                    }
                }
            }
    return ncube * 6;
}

/* ---------------------------------------------------------------------- */
/* Exact point-to-triangle squared distance (closest point by region,      */
/* C. Ericson, Real-Time Collision Detection, 2005, sec. 5.1.5).           */
/* ---------------------------------------------------------------------- */
static double pt_tri_d2(const double* p, const double* a, const double* b, const double* c)
{
    double ab[3], ac[3], ap[3];
    for (int i = 0; i < 3; ++i) { ab[i] = b[i] - a[i]; ac[i] = c[i] - a[i]; ap[i] = p[i] - a[i]; }
    const double d1 = ab[0] * ap[0] + ab[1] * ap[1] + ab[2] * ap[2];
    const double d2 = ac[0] * ap[0] + ac[1] * ap[1] + ac[2] * ap[2];
    double q[3];
    if (d1 <= 0.0 && d2 <= 0.0) { memcpy(q, a, sizeof q); goto out; }
    double bp[3];
    for (int i = 0; i < 3; ++i) bp[i] = p[i] - b[i];
    const double d3 = ab[0] * bp[0] + ab[1] * bp[1] + ab[2] * bp[2];
    const double d4 = ac[0] * bp[0] + ac[1] * bp[1] + ac[2] * bp[2];
    if (d3 >= 0.0 && d4 <= d3) { memcpy(q, b, sizeof q); goto out; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + v * ab[i];
        goto out;
    }
    double cp[3];
    for (int i = 0; i < 3; ++i) cp[i] = p[i] - c[i];
    const double d5 = ab[0] * cp[0] + ab[1] * cp[1] + ab[2] * cp[2];
    const double d6 = ac[0] * cp[0] + ac[1] * cp[1] + ac[2] * cp[2];
    if (d6 >= 0.0 && d5 <= d6) { memcpy(q, c, sizeof q); goto out; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + w * ac[i];
        goto out;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int i = 0; i < 3; ++i) q[i] = b[i] + w * (c[i] - b[i]);
        goto out;
    }
    {
        const double denom = 1.0 / (va + vb + vc);
        const double v = vb * denom, w = vc * denom;
        for (int i = 0; i < 3; ++i) q[i] = a[i] + ab[i] * v + ac[i] * w;
    }
out:;
    const double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}

/* Label tets by the unsigned distance of their centroid to a triangle mesh.
 * Centroid c (tet-vertex space) is mapped to query space by q = c*cs + co
 * per axis; mesh vertices are mapped by m = v*ms + mo.  labels[i] = 0 iff
 * dist(q, mesh) <= threshold.  Returns 0, or -1 on bad input. */
int synth_udf_labels(const double* V, int64_t nv, const int32_t* tets, int64_t N,
                     const double* cs, const double* co,
                     const double* TV, int64_t ntv, const int32_t* TF, int64_t ntf,
                     const double* ms, const double* mo,
                     double threshold, uint8_t* labels)
{
    if (ntf <= 0) { memset(labels, 1, (size_t)N); return 0; }
    double* MV = (double*)malloc((size_t)ntv * 3 * sizeof(double));
    if (!MV) return -1;
    double bmin[3] = {1e300, 1e300, 1e300}, bmax[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < ntv; ++i)
        for (int k = 0; k < 3; ++k) {
            const double m = TV[i * 3 + k] * ms[k] + mo[k];
            MV[i * 3 + k] = m;
            if (m < bmin[k]) bmin[k] = m;
            if (m > bmax[k]) bmax[k] = m;
        }
    /* grid over the threshold-expanded bbox; cell >= threshold */
    double span = 0.0;
    for (int k = 0; k < 3; ++k) {
        bmin[k] -= threshold;
        bmax[k] += threshold;
        if (bmax[k] - bmin[k] > span) span = bmax[k] - bmin[k];
    }
    double cell = span / 256.0;
    if (cell < threshold) cell = threshold;
    /* mean edge length keeps the triangle-per-cell fan-out small */
    double el = 0.0;
    int64_t nel = 0;
    const int64_t estep = ntf / 4096 + 1;
    for (int64_t f = 0; f < ntf; f += estep, ++nel) {
        const double* a = MV + (size_t)TF[f * 3] * 3;
        const double* b = MV + (size_t)TF[f * 3 + 1] * 3;
        el += sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
    }
    el /= (double)nel;
    if (cell < el) cell = el;
    int dim[3];
    for (int k = 0; k < 3; ++k) {
        dim[k] = (int)((bmax[k] - bmin[k]) / cell) + 1;
        if (dim[k] > 512) dim[k] = 512;
    }
    double inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = (double)dim[k] / (bmax[k] - bmin[k]);
    const int64_t ncell = (int64_t)dim[0] * dim[1] * dim[2];
    int64_t* off = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
    if (!off) { free(MV); return -1; }
    for (int pass = 0; pass < 2; ++pass) {
        int32_t* list = NULL;
        int64_t* fill = NULL;
        if (pass == 1) {
            for (int64_t c = 0; c < ncell; ++c) off[c + 1] += off[c];
            list = (int32_t*)malloc((size_t)off[ncell] * sizeof(int32_t) + 4);
            fill = (int64_t*)malloc((size_t)ncell * sizeof(int64_t));
            if (!list || !fill) { free(list); free(fill); free(off); free(MV); return -1; }
            memcpy(fill, off, (size_t)ncell * sizeof(int64_t));
        }
        for (int64_t f = 0; f < ntf; ++f) {
            int lo3[3], hi3[3];
            for (int k = 0; k < 3; ++k) {
                double mn = 1e300, mx = -1e300;
                for (int j = 0; j < 3; ++j) {
                    const double m = MV[(size_t)TF[f * 3 + j] * 3 + k];
                    if (m < mn) mn = m;
                    if (m > mx) mx = m;
                }
                lo3[k] = (int)floor((mn - threshold - bmin[k]) * inv[k]);
                hi3[k] = (int)floor((mx + threshold - bmin[k]) * inv[k]);
                if (lo3[k] < 0) lo3[k] = 0;
                if (hi3[k] >= dim[k]) hi3[k] = dim[k] - 1;
            }
            for (int z = lo3[2]; z <= hi3[2]; ++z)
                for (int y = lo3[1]; y <= hi3[1]; ++y)
                    for (int x = lo3[0]; x <= hi3[0]; ++x) {
                        const int64_t c = x + (int64_t)dim[0] * (y + (int64_t)dim[1] * z);
                        if (pass == 0) off[c + 1]++;
                        else list[fill[c]++] = (int32_t)f;
                    }
        }
        if (pass == 1) {
            free(fill);
            const double thr2 = threshold * threshold;
#pragma omp parallel for schedule(dynamic, 65536)
            for (int64_t i = 0; i < N; ++i) {
                double q[3] = {0.0, 0.0, 0.0};
                int bad = 0;
                for (int k = 0; k < 4; ++k) {
                    const int32_t vi = tets[i * 4 + k];
                    if (vi < 0 || vi >= nv) { bad = 1; break; }
                    q[0] += V[(size_t)vi * 3];
                    q[1] += V[(size_t)vi * 3 + 1];
                    q[2] += V[(size_t)vi * 3 + 2];
                }
                uint8_t lab = 1;
                if (!bad) {
                    int g[3], inside = 1;
                    for (int k = 0; k < 3; ++k) {
                        q[k] = (q[k] * 0.25) * cs[k] + co[k];
                        const double t = (q[k] - bmin[k]) * inv[k];
                        if (t < 0.0 || t >= (double)dim[k]) { inside = 0; break; }
                        g[k] = (int)t;
                    }
                    if (inside) {
                        const int64_t c = g[0] + (int64_t)dim[0] * (g[1] + (int64_t)dim[1] * g[2]);
                        for (int64_t e = off[c]; e < off[c + 1]; ++e) {
                            const int32_t f = list[e];
                            if (pt_tri_d2(q, MV + (size_t)TF[f * 3] * 3, MV + (size_t)TF[f * 3 + 1] * 3,
                                          MV + (size_t)TF[f * 3 + 2] * 3) <= thr2) { lab = 0; break; }
                        }
                    }
                }
                labels[i] = lab;
            }
            free(list);
        }
    }
    free(off);
    free(MV);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Narrow-band unsigned distance on a brick grid: the input of the tet-    */
/* centroid label sampler, standing in for OpenVDB's                       */
/* meshToUnsignedDistanceField (the reference's SparseUDF,                 */
/* native/vdb/wtivo_vdb.cpp:1007-1070, linear transform of voxel size h).  */
/* Voxel (i,j,k) sits at world (i,j,k)*h; a voxel closer than band to a    */
/* triangle holds its exact distance to the mesh (float), every other      */
/* voxel the background band.  Bricks are 8^3 voxels; the brick box is     */
/* [bmin3, bmin3 + dims) in brick units (voxel index >> 3).                */
/*   mode 0: mask[dims] = 1 for every brick a triangle's band box touches; */
/*   mode 1: values[brick][8][8][8] (z fastest, preset to the background   */
/*           by the caller) get the distances, through table[dims]         */
/*           (brick number, -1 = inactive).                                */
/* Returns 0, or -1 on a voxel outside the brick box.                      */
/* ---------------------------------------------------------------------- */
static void atomic_min_nonneg_float(float* p, float v)
{
    uint32_t nv_bits, old;
    memcpy(&nv_bits, &v, 4);
    uint32_t* q = (uint32_t*)p;
    old = __atomic_load_n(q, __ATOMIC_RELAXED);
    /* non-negative floats order like their bit patterns */
    while (nv_bits < old &&
           !__atomic_compare_exchange_n(q, &old, nv_bits, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}

int synth_brick_udf(const double* MV, int64_t nv, const int32_t* MF, int64_t nf, double h,
                    double band, const int32_t* bmin3, const int32_t* dims, int mode,
                    uint8_t* mask, const int32_t* table, float* values)
{
    (void)nv;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
    for (int64_t f = 0; f < nf; ++f) {
        const double* a = MV + (size_t)MF[f * 3] * 3;
        const double* b = MV + (size_t)MF[f * 3 + 1] * 3;
        const double* c = MV + (size_t)MF[f * 3 + 2] * 3;
        int64_t lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            double mn = a[k], mx = a[k];
            if (b[k] < mn) mn = b[k];
            if (c[k] < mn) mn = c[k];
            if (b[k] > mx) mx = b[k];
            if (c[k] > mx) mx = c[k];
            lo[k] = (int64_t)ceil((mn - band) / h);
            hi[k] = (int64_t)floor((mx + band) / h);
        }
        for (int k = 0; k < 3; ++k)
            if ((lo[k] >> 3) < bmin3[k] || (hi[k] >> 3) >= (int64_t)bmin3[k] + dims[k]) bad = 1;
        if (bad) continue;
        if (mode == 0) {
            for (int64_t x = lo[0] >> 3; x <= hi[0] >> 3; ++x)
                for (int64_t y = lo[1] >> 3; y <= hi[1] >> 3; ++y)
                    for (int64_t z = lo[2] >> 3; z <= hi[2] >> 3; ++z)
                        mask[((x - bmin3[0]) * dims[1] + (y - bmin3[1])) * dims[2] + (z - bmin3[2])] = 1;
            continue;
        }
        for (int64_t x = lo[0]; x <= hi[0]; ++x)
            for (int64_t y = lo[1]; y <= hi[1]; ++y)
                for (int64_t z = lo[2]; z <= hi[2]; ++z) {
                    const double p[3] = {(double)x * h, (double)y * h, (double)z * h};
                    const double d = sqrt(pt_tri_d2(p, a, b, c));
                    if (!(d < band)) continue;
                    const int64_t bi = ((((x >> 3) - bmin3[0]) * dims[1] + ((y >> 3) - bmin3[1])) * dims[2] +
                                        ((z >> 3) - bmin3[2]));
                    const int32_t brick = table[bi];
                    if (brick < 0) continue;
                    atomic_min_nonneg_float(values + (size_t)brick * 512 + ((x & 7) * 8 + (y & 7)) * 8 + (z & 7),
                                            (float)d);
                }
    }
    return bad ? -1 : 0;
}

/*
 * synth_raw_graph: the integer-capacity raw graph of a tet mesh (all cells
 * free, CelloCut slots).  n-link of slot k of tet i = rint(scale * area /
 * mean_area) (scale 1e4 in the integer-graph workload), where area is the
 * face's area taken from the face's lower-id
 * tet, so both directions of a face carry the same capacity, and mean_area
 * is the mean over every slot with a neighbour.  t-links from the signed
 * distance of the centroid (mean of the 4 vertices) to the sphere of centre
 * (0.5,0.5,0.5) and radius 0.3 plus noise[i]: src = rint(100 max(0, -d)),
 * snk = rint(100 max(0, d)).  area_scratch holds 4N doubles.  Sums run over
 * fixed blocks in a fixed order, so the result does not depend on the thread
 * count.  Returns 0, or -1 when a neighbour does not list the tet back.
 */
int synth_raw_graph(const double* P, const int32_t* tets, const int32_t* nbrs, int64_t N,
                    const double* noise, double scale, double* area_scratch, uint32_t* cap,
                    uint32_t* src, uint32_t* snk)
{
    static const int lut[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int64_t BLK = 65536;
    const int64_t nblk = (N + BLK - 1) / BLK;
    double* bsum = (double*)calloc((size_t)(nblk > 0 ? nblk : 1), sizeof(double));
    int64_t* bcnt = (int64_t*)calloc((size_t)(nblk > 0 ? nblk : 1), sizeof(int64_t));
    if (!bsum || !bcnt) { free(bsum); free(bcnt); return -2; }
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nblk; ++b) {
        double s = 0.0;
        int64_t c = 0;
        const int64_t e = (b + 1) * BLK < N ? (b + 1) * BLK : N;
        for (int64_t i = b * BLK; i < e; ++i) {
            for (int f = 0; f < 4; ++f) {
                const double* a = P + 3 * (int64_t)tets[4 * i + lut[f][0]];
                const double* q = P + 3 * (int64_t)tets[4 * i + lut[f][1]];
                const double* r = P + 3 * (int64_t)tets[4 * i + lut[f][2]];
                const double u0 = q[0] - a[0], u1 = q[1] - a[1], u2 = q[2] - a[2];
                const double v0 = r[0] - a[0], v1 = r[1] - a[1], v2 = r[2] - a[2];
                const double c0 = u1 * v2 - u2 * v1, c1 = u2 * v0 - u0 * v2, c2 = u0 * v1 - u1 * v0;
                const double ar = 0.5 * sqrt(c0 * c0 + c1 * c1 + c2 * c2);
                area_scratch[4 * i + f] = ar;
                if (nbrs[4 * i + f] >= 0) { s += ar; ++c; }
            }
        }
        bsum[b] = s;
        bcnt[b] = c;
    }
    double total = 0.0;
    int64_t count = 0;
    for (int64_t b = 0; b < nblk; ++b) { total += bsum[b]; count += bcnt[b]; }
    free(bsum);
    free(bcnt);
    const double mean = count ? total / (double)count : 1.0;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < N; ++i) {
        for (int f = 0; f < 4; ++f) {
            const int32_t j = nbrs[4 * i + f];
            if (j < 0) { cap[4 * i + f] = 0u; continue; }
            double fa = area_scratch[4 * i + f];
            if ((int64_t)j < i) {
                int rk = -1;
                for (int k = 0; k < 4; ++k)
                    if (nbrs[4 * (int64_t)j + k] == (int32_t)i) rk = k;
                if (rk < 0) { bad = 1; rk = 0; }
                fa = area_scratch[4 * (int64_t)j + rk];
            }
            cap[4 * i + f] = (uint32_t)rint(scale * fa / mean);
        }
        double c[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < 4; ++k)
            for (int a = 0; a < 3; ++a) c[a] += P[3 * (int64_t)tets[4 * i + k] + a];
        const double dx = 0.25 * c[0] - 0.5, dy = 0.25 * c[1] - 0.5, dz = 0.25 * c[2] - 0.5;
        const double d = sqrt(dx * dx + dy * dy + dz * dz) - 0.3 + noise[i];
        src[i] = (uint32_t)rint(100.0 * (d < 0.0 ? -d : 0.0));
        snk[i] = (uint32_t)rint(100.0 * (d > 0.0 ? d : 0.0));
    }
    return bad ? -1 : 0;
}
