/*
 * wtivo_oracle.h -- CPU oracle for the WTiVo graph-cut hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product is compared against; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it.  The product never calls it and
 * has no CPU fallback.
 *
 * It restates, in plain C, the reference's semantics for:
 *   - reduced-graph build: classification + compaction
 *     (native/gpupr/wtivo_gpupr_bindings.cpp:146-188), per-direction
 *     capacity formula (:65-98), ELL rows, t-links, terminal base flow
 *     (:227-314);
 *   - Phase-I push-relabel as a sequential FIFO restatement of
 *     native/gpupr/gpu_push_relabel_fast.cu:406-571 (exact global relabel
 *     :360-402, discharge rules :185-313, final BFS + partition :551-562);
 *   - an independent Boykov-Kolmogorov max flow (Boykov & Kolmogorov,
 *     IEEE PAMI 26(9), 2004) used as the exactness oracle;
 *   - the sink-reachable partition (.cu:315-324) and the label scatter
 *     (bindings.cpp:357-364);
 *   - the cut-surface extraction (bindings.cpp:400-577).
 *
 * All capacities are integers (the reference truncates float areas to
 * int32), so every flow here is exact int64 arithmetic.
 */
#ifndef WTIVO_ORACLE_H
#define WTIVO_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_ERR_ARG = 1,          /* bad argument / size */
    ORC_ERR_NBR_RANGE = 2,    /* neighbor index >= N ("neighbor out of range") */
    ORC_ERR_REFS_ODD = 3,     /* "neighbor reference count not even" */
    ORC_ERR_BUILD = 4,        /* "invalid graph reduction/capacity state" */
    ORC_ERR_FREE_REFS_ODD = 5,/* "free reference count not even" */
    ORC_ERR_TOO_MANY = 6,     /* ">INT32_MAX reduced nodes unsupported" */
    ORC_ERR_NO_REVERSE = 7,   /* asymmetric adjacency: reverse slot missing */
    ORC_ERR_NO_MEM = 8,
    ORC_ERR_MAX_ROUNDS = 9,
    ORC_ERR_INVARIANT = 10,   /* active node without residual out-arc */
    ORC_ERR_NEG_VERTEX = 11,  /* "negative vertex index" (wtivo_core.cpp:424) */
    ORC_ERR_BBOX = 12,        /* "...sample_tet_labels: degenerate bbox" (wtivo_vdb.cpp:1547) */
    ORC_ERR_TET_INDEX = 13    /* "...sample_tet_labels: tet index out of range" (:1566) */
};

typedef struct {
    uint64_t n_full;          /* N */
    uint64_t free_n;          /* F */
    uint64_t fixed_source;    /* label == 0 */
    uint64_t fixed_sink;      /* label != 0 and a -1 neighbor */
    uint64_t full_refs;       /* non-negative neighbor entries over all tets */
    uint64_t free_refs;       /* free->free arcs */
    uint64_t terminal_edges;  /* free->fixed arcs */
    int64_t terminal_base_flow; /* sum over free nodes of min(src, snk) */
} orc_build_info;

/* Capacity of the arc leaving face slot fi of tet `tet4` toward a tet with
 * label lj, the tet itself having label li (bindings.cpp:65-98).
 * Returns ORC_OK or ORC_ERR_BUILD (invalid vertex / capacity out of range). */
int orc_capacity(const double* V, uint64_t nv, const int32_t* tet4, int fi,
                 uint8_t li, uint8_t lj, double fill_T, int32_t* cap);

/* Classification + compaction (bindings.cpp:146-188).
 * full_to_free[N]: reduced id, -2 fixed source, -3 fixed sink.
 * free_old[N] (capacity N): original tet index of each reduced node. */
int orc_classify(const int32_t* nbrs, const uint8_t* labels, uint64_t N,
                 int32_t* full_to_free, uint32_t* free_old,
                 orc_build_info* info);

/* Reduced ELL graph (bindings.cpp:227-314). Arrays sized by info->free_n:
 * nbr[4F] (reduced id or -1), res[4F], term[F] = src - snk. */
int orc_build(const double* V, uint64_t nv, const int32_t* tets,
              const int32_t* nbrs, const uint8_t* labels, uint64_t N,
              double fill_T, const int32_t* full_to_free,
              orc_build_info* info, int32_t* nbr, uint32_t* res,
              int32_t* term);

/* Reverse slot of every arc: rev[4F] in {0..3}, 255 for empty slots. */
int orc_reverse_slots(uint32_t F, const int32_t* nbr, uint8_t* rev);

/* Boykov-Kolmogorov max flow on the reduced ELL graph.
 * res/term are updated in place to the final residual graph (term<0:
 * remaining sink capacity; term>0: remaining source capacity).
 * partition[F] = 1 iff the node reaches the sink in the residual graph. */
int orc_maxflow_bk(uint32_t F, const int32_t* nbr, uint32_t* res,
                   int32_t* term, int64_t* raw_flow, uint8_t* partition);

/* Sequential Phase-I push-relabel with the reference's rules.
 * excess[F] receives the final preflow excess; term is updated like the
 * reference's d_terminal (sink pushes raise negative terms toward 0).
 * rounds/relabels (optional) receive discharge passes and global relabels. */
int orc_maxflow_pr(uint32_t F, const int32_t* nbr, uint32_t* res,
                   int32_t* term, int64_t* excess, int local_steps,
                   int global_relabel_period, uint64_t max_rounds,
                   int64_t* raw_flow, uint8_t* partition,
                   uint64_t* rounds, uint64_t* relabels);

/* partition[v] = 1 iff v reaches the sink through residual arcs
 * (term<0 is a residual arc to the sink). */
int orc_sink_reachable(uint32_t F, const int32_t* nbr, const uint32_t* res,
                       const int32_t* term, uint8_t* partition);

/* Whole graph_cut_fast path: build, BK solve, scatter.
 * out_labels[N]; stats[8] = {adjusted_flow, raw_flow, full_E, free_E,
 * fixed_source, fixed_sink, terminal_edges, free_n}. solver: 0 = BK,
 * 1 = sequential push-relabel. */
int orc_graph_cut(const double* V, uint64_t nv, const int32_t* tets,
                  const int32_t* nbrs, const uint8_t* labels, uint64_t N,
                  double fill_T, int solver, uint8_t* out_labels,
                  int64_t* stats);

/* Cut-surface extraction (bindings.cpp:400-577).  The reference's
 * par_chunks ranges are contiguous and concatenated in thread order, so its
 * face order is plain tet order, then slot order; the thread count does not
 * change it.  Two calls: with out_faces==NULL only the counts are returned;
 * then with buffers of those sizes.  out_faces[3*faces] holds compacted
 * vertex ids, out_verts[3*used] the used vertices in original order. */
int orc_surface(const uint8_t* labels, const double* V, uint64_t nv,
                const int32_t* tets, const int32_t* nbrs, uint64_t N,
                uint64_t* n_faces, uint64_t* n_used,
                int32_t* out_faces, double* out_verts);

/* Edge-degree watertight audit (native/core/wtivo_core.cpp:402-464): every
 * face contributes its three undirected edges as keys (min << 32 | max),
 * the keys are sorted, and each run of equal keys whose length is not 2 is
 * one bad edge group.  A closed 2-manifold mesh has none.  Returns ORC_OK or
 * ORC_ERR_NEG_VERTEX.  The reference function needs CGAL/TBB to build; its
 * own known-answer case (scripts/verify_install.py:38-41, a tetrahedron
 * shell: watertight, 0 bad groups) pins this restatement in the tests.
 * Parity of the label sampler below is unpinned: it follows OpenVDB's
 * published BoxSampler, and no OpenVDB is present to compare against. */
int orc_edge_audit(const int32_t* faces, uint64_t nf, uint64_t* bad_groups);

/* Sparse unsigned distance grid of 8^3-voxel bricks (host arrays): voxel
 * (i,j,k) sits at world (i,j,k)*voxel_size; brick (bx,by,bz) of the box
 * holds voxels origin + 8*(bx,by,bz) + [0,8)^3; table[(bx*dims[1]+by)*dims[2]+bz]
 * is the brick's number in values (-1: every voxel = background);
 * values[brick*512 + (x*8+y)*8+z]. */
typedef struct {
    double voxel_size;
    int32_t origin[3];
    int32_t dims[3];
    float background;
    const int32_t* table;
    const float* values;
} orc_brick_grid;

/* Tet-centroid labels (native/vdb/wtivo_vdb.cpp:1519-1584,
 * SparseUDF.sample_tet_labels): centroid = 0.25 * sum of the 4 vertices,
 * mapped into the query box n = ((c - bmin)/(bmax - bmin))*(1 - 2 padding)
 * + padding, to index space by the grid's linear transform (n * (1/h)),
 * sampled by OpenVDB 12.0.1's BoxSampler (trilinear over the 8 voxels
 * around floor(index): lerp along z, then y, then x, each lerp
 * a + float((b - a) * w)); label 0 where the sample <= threshold, else 1.
 * udf (optional) receives the samples. */
int orc_sample_tet_labels(const orc_brick_grid* g, const double* V, uint64_t nv,
                          const int32_t* tets, uint64_t nt, const double* bmin,
                          const double* bmax, double padding, double threshold,
                          uint8_t* labels, float* udf);

#ifdef __cplusplus
}
#endif
#endif
