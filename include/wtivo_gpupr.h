/*
 * wtivo_gpupr.h -- C ABI of the B200 graph-cut library (libwtivo_gpupr.so).
 *
 * The min s-t cut over the Delaunay tet cell graph of WTiVo: reduced-graph
 * build, multi-discharge push-relabel with exact global relabels, and the
 * final residual BFS that fixes the source/sink partition.  Plain pointers
 * and sizes only; no exceptions cross this boundary; every entry point
 * returns a gpupr_status and keeps a human-readable detail message that
 * gpupr_last_error() returns (per thread).
 *
 * Streams: `stream` is a cudaStream_t passed as void* (NULL = the legacy
 * default stream).  Calls return after their results are complete.
 */
#ifndef WTIVO_GPUPR_H
#define WTIVO_GPUPR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPUPR_ABI_VERSION 6   /* 2: stats and options carry the persistent engine's
                                 grid, relabel factor and chaining; tuning entries.
                                 3: stats carry the active-sweep time, the graphs
                                 a batch retired early and the bottom-up steps;
                                 options carry the direction-optimizing BFS switch.
                                 4: options carry relabel_tiles, stats the tile
                                 steps (53 eight-byte stats fields).
                                 5: options carry bfs_block_levels and
                                 bfs_in_arc_masks.
                                 6: stats carry the discharge rounds and their
                                 time by active-set size (59 eight-byte stats
                                 fields) */

typedef enum {
    GPUPR_OK = 0,
    GPUPR_ERR_INVALID_ARGUMENT = 1,  /* shapes/pointers (bindings.cpp:114-133) */
    GPUPR_ERR_NEIGHBOR_RANGE = 2,    /* "neighbor out of range" (bindings.cpp:172) */
    GPUPR_ERR_REFS_ODD = 3,          /* "neighbor reference count not even" (:177) */
    GPUPR_ERR_BUILD = 4,             /* "invalid graph reduction/capacity state" (:297) */
    GPUPR_ERR_FREE_REFS_ODD = 5,     /* "free reference count not even" (:318) */
    GPUPR_ERR_TOO_MANY_NODES = 6,    /* ">INT32_MAX reduced nodes unsupported" (:198) */
    GPUPR_ERR_NO_REVERSE = 7,        /* asymmetric adjacency (.cu:129,254 codes 2/4) */
    GPUPR_ERR_OUT_OF_MEMORY = 8,     /* "insufficient VRAM ..." (:212) */
    GPUPR_ERR_MAX_ROUNDS = 9,        /* "max macro rounds exceeded" (.cu:492) */
    GPUPR_ERR_INVARIANT = 10,        /* device invariant failed (.cu:206,292) */
    GPUPR_ERR_CUDA = 11,             /* CUDA runtime failure (.cu:23-29) */
    GPUPR_ERR_TIMEOUT = 12,          /* solve time limit (.cu:542-543) / bounded wait */
    GPUPR_ERR_TOO_MANY_TETS = 13     /* ">2^32 full tets unsupported" (:132) */
} gpupr_status;

/* Statistics of one graph_cut call.  The first 18 fields are the 18-tuple of
 * graph_cut_fast (bindings.cpp:377-396) in order. */
typedef struct {
    int64_t adjusted_flow;      /* raw_flow + terminal base flow */
    int64_t raw_flow;           /* flow pushed into the sink by the solver */
    uint64_t graph_bytes;       /* device bytes of the reduced graph */
    uint64_t workspace_bytes;   /* device bytes of the solver workspace */
    uint64_t full_E;            /* faces between finite tets */
    uint64_t free_E;            /* faces between free tets */
    uint64_t fixed_source;
    uint64_t fixed_sink;
    uint64_t terminal_edges;
    int64_t threads;            /* echoed max(1, threads) */
    uint64_t rounds;            /* discharge rounds */
    uint64_t global_relabels;   /* exact BFS relabels, the final one included */
    uint64_t map_bytes;         /* N*4 + F*4 */
    double build_seconds;       /* classify + reduced-graph build */
    int64_t local_steps;        /* echoed as passed */
    double solve_seconds;       /* push-relabel until the active set is empty */
    double native_total_seconds;
    /* extensions */
    uint64_t free_n;
    uint64_t n_full;
    double final_relabel_seconds;
    double partition_seconds;
    uint64_t node_visits;       /* discharge node visits */
    uint64_t pushes;            /* arc pushes (sink pushes included) */
    uint64_t bfs_visits;        /* frontier nodes expanded by BFS levels */
    uint64_t bfs_levels;        /* BFS levels over all global relabels */
    uint64_t kernel_launches;   /* kernels this call launched */
    double solve_device_ms;     /* CUDA-event time of the solve phase */
    double build_device_ms;     /* CUDA-event time of the build phase */
    double discharge_ms;        /* CUDA-event time of all discharge batches */
    double bfs_ms;              /* CUDA-event time of all global-relabel BFS */
    uint64_t discharge_launches;
    uint64_t bfs_launches;
    int64_t engine;             /* 1 one launch per step, 2 persistent */
    int64_t solve_blocks_per_sm;/* persistent engine: resident blocks per SM used */
    double relabel_work_factor; /* persistent engine: relabel work factor used */
    int64_t chain_hops;         /* persistent engine: chained discharge used */
    int64_t chain_max_active;
    double sweep_ms;            /* persistent engine: active sweeps after each relabel
                                   (part of bfs_ms) */
    uint64_t graphs_retired;    /* batch: graphs finished and left out of the
                                   relabels before the last one */
    uint64_t bottom_up_steps;   /* BFS steps run bottom-up (bfs_bottom_up) */
    uint64_t bfs_steps_by_frontier[3];  /* persistent engine: BFS steps over frontiers
                                           of <= 1024, <= 16384 and more nodes */
    double bfs_ms_by_frontier[3];       /* ... and their time (block 0's clock) */
    uint64_t bfs_tail_steps;    /* BFS steps run by one block (bfs_tail_max) */
    uint64_t bfs_tail_levels;   /* ... and the levels they covered */
    int64_t relabel_tiles;      /* persistent engine: 1 = the relabels ran by tiles */
    uint64_t tile_steps;        /* tiled relabels: tile steps (grid barriers) */
    uint64_t tile_procs;        /* ... tiles processed */
    uint64_t tile_loads;        /* ... nodes those tiles loaded */
    uint64_t tile_writes;       /* ... labels lowered */
    uint64_t discharge_rounds_by_active[3]; /* persistent engine: discharge rounds
                                           over <= 4096, <= 131072 and more
                                           active nodes */
    double discharge_ms_by_active[3];       /* ... and their time (block 0's clock) */
} gpupr_cut_stats;

/* Solver tuning knobs; zero fields take the defaults shown. */
typedef struct {
    int32_t local_steps;          /* 1..32, default 8 */
    int32_t global_relabel_period;/* default 1024; one-launch-per-step engine:
                                     relabel every ceil(period/local_steps)
                                     rounds (gpu_push_relabel_fast.cu:476-480);
                                     persistent engine: at most `period`
                                     rounds between relabels; < 0 = no cap */
    uint64_t max_rounds;          /* default 2,000,000 */
    double time_limit_seconds;    /* default 240 */
    int32_t round_batch;          /* rounds enqueued per host check, default 24 */
    int32_t bfs_batch;            /* BFS levels enqueued per host check, default 48 */
    int32_t block_size;           /* threads per block, default 256 */
    int32_t blocks_per_sm;        /* resident blocks per SM; default: 4 (one
                                     launch per step), by graph size 2..4
                                     (persistent: 2 below 1.5M free nodes, 3
                                     below 5M, else 4) */
    double work_relabel_factor;   /* relabel after this many node visits per
                                     free node since the last one; default 3
                                     (one launch per step); persistent: 2 below
                                     500k free nodes, 1 below 10M, else 0.5 */
    int32_t engine;               /* 0 auto (persistent when the device supports
                                     cooperative launch), 1 one launch per BFS
                                     level / round, 2 persistent */
    int32_t chain_hops;           /* persistent engine: nodes one thread may
                                     discharge in a row in one round (1 = no
                                     chaining; default 4) */
    int32_t chain_max_active;     /* ... only in rounds with at most this many
                                     active nodes (default by graph size: 131072
                                     below 1.5M free nodes, 32768 below 2M,
                                     else 4096) */
    int32_t bfs_bottom_up;        /* persistent engine: 1 = direction-optimizing
                                     global relabels (bottom-up steps over the
                                     nodes the previous relabel reached and this
                                     one has not, once they number at most
                                     bfs_bottom_up_ratio x the frontier);
                                     0 = top-down only (default) */
    double bfs_bottom_up_ratio;   /* default 1 */
    int32_t bfs_chain_hops;       /* persistent engine: nodes one thread may label
                                     in a row in a BFS step over a short frontier
                                     (1 = level by level; default 4) */
    int32_t bfs_tail_max;         /* persistent engine: a BFS frontier of at most
                                     this many nodes (up to 1024) is expanded by
                                     one block alone, level after level, with
                                     block-level syncs (0 = default, < 0 = never) */
    int32_t discharge_warp_aggregate; /* persistent engine: 1 = lanes of a warp that
                                     push to the same neighbour add their amounts
                                     with one atomic (default 0: one atomic each) */
    int32_t bfs_chain_max_frontier; /* persistent engine: BFS steps chain
                                     (bfs_chain_hops) only over frontiers of at
                                     most this many nodes (default: any frontier
                                     whose chained step fits the queue bound) */
    int32_t relabel_tiles;        /* persistent engine: 1 = global relabels by
                                     tiles of 2048 consecutive nodes, each
                                     solved in shared memory and re-run when a
                                     label it reads from another tile goes
                                     down (exact distances, no in-arc rows);
                                     < 0 = frontier steps; 0 = default (frontier
                                     steps); bfs_bottom_up and bfs_tail_max
                                     apply to frontier steps only */
    int32_t bfs_block_levels;     /* persistent engine: each BFS step expands its
                                     frontier and then, per block and without a
                                     grid barrier, up to this many levels in all
                                     from the nodes the block labelled itself
                                     (breadth first, shared-memory stage);
                                     0 = default (16), 1 = per-thread chains
                                     instead (bfs_chain_hops, bfs_chain_max_frontier) */
    int32_t bfs_in_arc_masks;     /* persistent engine, frontier steps: 1 = each
                                     relabel's seed sweep writes one byte per node
                                     (which neighbours have a residual arc into
                                     it) and a BFS step reads the node's
                                     neighbour row with it; < 0 = the sweep writes
                                     a 16-byte in-arc row per node instead;
                                     0 = default */
} gpupr_solve_options;

const char* gpupr_status_string(gpupr_status status);
const char* gpupr_last_error(void);
int gpupr_abi_version(void);

/*
 * Whole graph_cut_fast path.
 * Replaces graph_cut_gpupr_fast_v630 (native/gpupr/wtivo_gpupr_bindings.cpp:
 * 100-397) behind wtivo_gpupr.graph_cut_fast (:581-590).
 *   vertices   float64 [n_vertices*3]   host (vertices_on_device=0) or device
 *   d_tets     int32   [n_tets*4]        device
 *   d_neighbors int32  [n_tets*4]        device, CelloCut slots, -1 = hull
 *   labels     uint8   [n_tets]          host or device
 *   out_labels uint8   [n_tets]          host or device: input labels with
 *              every free tet replaced by 1 iff it reaches the sink
 * threads is only echoed in the stats (the build runs on the GPU).
 * local_steps, global_relabel_period and max_rounds keep the reference's
 * meaning and clamps (gpu_push_relabel_fast.cu:421-424,476-480).
 * When no tet is free the output equals the input labels and
 * stats->free_n == 0 (bindings.cpp:191-196).
 */
gpupr_status gpupr_graph_cut(const double* vertices, uint64_t n_vertices,
                             int vertices_on_device, const int32_t* d_tets,
                             const int32_t* d_neighbors, uint64_t n_tets,
                             const uint8_t* labels, int labels_on_device,
                             double fill_T, int32_t threads,
                             int32_t global_relabel_period, uint64_t max_rounds,
                             int32_t local_steps, uint8_t* out_labels,
                             int out_on_device, void* stream,
                             gpupr_cut_stats* stats);

/* Same as gpupr_graph_cut with explicit solver options (NULL = defaults). */
gpupr_status gpupr_graph_cut_ex(const double* vertices, uint64_t n_vertices,
                                int vertices_on_device, const int32_t* d_tets,
                                const int32_t* d_neighbors, uint64_t n_tets,
                                const uint8_t* labels, int labels_on_device,
                                double fill_T, int32_t threads,
                                const gpupr_solve_options* options,
                                uint8_t* out_labels, int out_on_device,
                                void* stream, gpupr_cut_stats* stats);

/* One graph of a batch: its flows and sizes. */
typedef struct {
    int64_t adjusted_flow;   /* max flow of this graph (raw + terminal base flow) */
    int64_t raw_flow;
    uint64_t n_tets;
    uint64_t free_n;
} gpupr_batch_item;

/*
 * Batched graph cut: n_graphs independent cell graphs cut in one solve.
 * No counterpart in the reference (it cuts one graph per call).  The graphs
 * are packed end to end: graph g owns tets [tet_offsets[g], tet_offsets[g+1])
 * and vertices [vertex_offsets[g], vertex_offsets[g+1]) of the concatenated
 * arrays, and its tets/neighbors use LOCAL ids (0-based within the graph,
 * -1 = hull), exactly what graph_cut_fast takes for one graph.  Offsets are
 * host arrays of n_graphs+1 entries starting at 0.  out_labels is the
 * concatenation of every graph's graph_cut_fast labels; items[g] receives
 * each graph's flows.  One fill_T and one set of options for the batch.
 * The union is solved as segments: each graph retires once a global relabel
 * finds no active node in it (its labels are then final and later relabels
 * skip it).  Unless options set chain_hops, chain_max_active, blocks_per_sm or
 * work_relabel_factor, the batch takes the batch tuning table's entry for its
 * size bucket (gpupr_autotune_batch); without one, a batch of at least 16
 * graphs averaging under 1.5M tets solves with 8 chained hops in rounds of up
 * to 131072 active nodes on 3 blocks per SM (the setting that suits small
 * graphs; the union's own size would pick another).
 */
gpupr_status gpupr_graph_cut_batch(uint32_t n_graphs, const uint64_t* tet_offsets,
                                   const uint64_t* vertex_offsets, const double* vertices,
                                   int vertices_on_device, const int32_t* d_tets,
                                   const int32_t* d_neighbors, const uint8_t* labels,
                                   int labels_on_device, double fill_T,
                                   const gpupr_solve_options* options, uint8_t* out_labels,
                                   int out_on_device, void* stream, gpupr_batch_item* items,
                                   gpupr_cut_stats* stats);

/*
 * Serving loop (continuous batching).  No counterpart in the reference.
 * A server owns, per lane, two threads on the device current at creation: a
 * stager that admits the lane's requests in arrival order while their
 * estimated device footprint fits hbm_budget_bytes (0 = 160 GiB) next to
 * every batch staged or being solved and uploads them as one packed batch,
 * and a solver that cuts each staged batch in one solve.  Requests that
 * arrive while a batch runs join the lane's next one.
 * A request is one cell graph in HOST arrays with graph_cut_fast's layout;
 * the server BORROWS them (no copy): vertices, tets, neighbors and labels
 * must stay valid and unchanged, and out_labels (n_tets bytes) writable,
 * until gpupr_server_wait() has returned for the request or the server is
 * destroyed (destroy finishes every submitted request first).
 */
typedef struct gpupr_server gpupr_server;
typedef struct {
    uint64_t id;
    int32_t status;           /* gpupr_status of the request */
    int32_t batch_size;       /* requests cut in the same batch */
    int64_t adjusted_flow;
    int64_t raw_flow;
    uint64_t n_tets;
    uint64_t free_n;
    double queue_ms;          /* submit -> admitted into a batch */
    double upload_ms;         /* the batch's host -> device copies */
    double solve_ms;          /* the batch's cut, labels copied out */
    double latency_ms;        /* submit -> result ready */
    int32_t lane;             /* 0 small-request lane, 1 large-request lane */
    int32_t reserved;
} gpupr_request_result;

/* max_batch: most requests per batch and lane (0 = no limit; 1 = one request
 * at a time per lane, uploads still overlapping the previous cut).
 * gpupr_server_create splits requests at 2,000,000 tets into two lanes whose
 * solves run at the same time: requests below the split go to the small lane
 * (its persistent grid capped at 1 resident block per SM), the rest to the
 * large lane (capped at the solver kernel's occupancy limit minus one), so
 * both lanes' grids are resident together and a small request never waits
 * for a large one's solve.  A small request submitted while the small lane
 * has work in flight and the large lane has none takes the large lane
 * (gpupr_request_result.lane says which).  The HBM budget covers both lanes.
 * gpupr_server_create_lanes takes the split; split_tets = 0 gives one lane
 * (every solve on the whole GPU, one at a time). */
gpupr_status gpupr_server_create(uint64_t hbm_budget_bytes, uint32_t max_batch,
                                 const gpupr_solve_options* options, gpupr_server** server);
gpupr_status gpupr_server_create_lanes(uint64_t hbm_budget_bytes, uint32_t max_batch,
                                       const gpupr_solve_options* options, uint64_t split_tets,
                                       gpupr_server** server);
gpupr_status gpupr_server_submit(gpupr_server* server, const double* vertices,
                                 uint64_t n_vertices, const int32_t* tets,
                                 const int32_t* neighbors, const uint8_t* labels,
                                 uint64_t n_tets, double fill_T, uint8_t* out_labels,
                                 uint64_t* request_id);
/* Blocks until the request is done (or timeout_s, > 0, passes; the request
 * then stays in flight), fills result and releases the request: its labels
 * are in the out_labels array given at submit. */
gpupr_status gpupr_server_wait(gpupr_server* server, uint64_t request_id, double timeout_s,
                               gpupr_request_result* result);
gpupr_status gpupr_server_destroy(gpupr_server* server);

/*
 * Reduced-graph build only (bindings.cpp:146-314): writes the reference's
 * host arrays so the build can be compared byte for byte.  All outputs are
 * HOST buffers sized by the caller: full_to_free[n_tets], free_old[n_tets],
 * nbr[4*n_tets], res[4*n_tets], term[n_tets], rev[n_tets] (2-bit reverse
 * slots, slot k in bits 2k..2k+1).  info[8] = {free_n, fixed_source,
 * fixed_sink, full_refs, free_refs, terminal_edges, terminal_base_flow,
 * n_tets}.
 */
gpupr_status gpupr_build_reduced(const double* vertices, uint64_t n_vertices,
                                 int vertices_on_device, const int32_t* d_tets,
                                 const int32_t* d_neighbors, uint64_t n_tets,
                                 const uint8_t* labels, int labels_on_device,
                                 double fill_T, int32_t* full_to_free,
                                 uint32_t* free_old, int32_t* nbr, uint32_t* res,
                                 int32_t* term, uint8_t* rev, int64_t* info,
                                 void* stream);

/*
 * Phase-I solve of a reduced graph already in device memory.
 * Replaces cellocut_gpu_push_relabel_fast
 * (native/gpupr/gpu_push_relabel_fast.h:20-28, .cu:406-571): same layout
 * (d_neighbors int32[4n], d_residual uint32[4n], d_terminal int32[n], both
 * updated in place to the final residual graph), h_partition uint8[n] on the
 * host (1 = reaches the sink).  d_excess_out (optional, device int64[n])
 * receives the final preflow excess.
 */
gpupr_status gpupr_solve_reduced(uint32_t n, int32_t* d_neighbors,
                                 uint32_t* d_residual, int32_t* d_terminal,
                                 uint8_t* h_partition,
                                 int32_t global_relabel_period,
                                 uint64_t max_rounds, int32_t local_steps,
                                 int64_t* d_excess_out, void* stream,
                                 gpupr_cut_stats* stats);

/*
 * Raw-graph entry (no reduction): every node is free, n-links cap[4n] in
 * CelloCut ELL slots (nbr -1 = none), source capacities src[n] and sink
 * capacities snk[n].  All inputs are DEVICE buffers and are not modified.
 * Outputs: *max_flow (host) and d_partition uint8[n] (device, 1 = reaches
 * the sink; the minimal sink side of the minimum cut).  No reference
 * counterpart: it serves integer-capacity graphs that do not come from
 * graph_cut_fast's reduction.
 */
gpupr_status gpupr_solve_ell(uint32_t n, const int32_t* d_nbr,
                             const uint32_t* d_cap, const uint32_t* d_src,
                             const uint32_t* d_snk,
                             const gpupr_solve_options* options,
                             int64_t* max_flow, uint8_t* d_partition,
                             void* stream, gpupr_cut_stats* stats);

/*
 * Cut-surface extraction.  Replaces surface_extraction_topology_cuda
 * (bindings.cpp:400-577): the oriented boundary faces of label-0 tets in the
 * reference's order, with vertices compacted in original order.  Two-step:
 * gpupr_surface_count() returns the face and used-vertex counts and keeps the
 * result on the device for the next gpupr_surface_fetch() on the same
 * thread.  labels and vertices are host or device; tets/neighbors device.
 */
gpupr_status gpupr_surface_count(const uint8_t* labels, int labels_on_device,
                                 const double* vertices, uint64_t n_vertices,
                                 int vertices_on_device, const int32_t* d_tets,
                                 const int32_t* d_neighbors, uint64_t n_tets,
                                 uint64_t* n_faces, uint64_t* n_used,
                                 void* stream);
gpupr_status gpupr_surface_fetch(int32_t* faces, double* vertices_out,
                                 int out_on_device, void* stream);

/*
 * Allocation-free variant of gpupr_solve_reduced.  No counterpart in the
 * reference.  For callers that cannot allocate device memory during the call:
 * an application whose own allocator already owns the device heap, or code
 * that must not enter the CUDA allocator mid-pipeline.  Nothing is allocated
 * on the device or the host on success: the solver's scratch (reverse slots,
 * arc-pair residual sums, excess, heights, queues, control block; about
 * 41 MiB) is a static device array inside this library, which every GPU that
 * loads the library's solver module holds until the process exits.
 *   n            at most 1,048,576 nodes; larger graphs are rejected with
 *                GPUPR_ERR_INVALID_ARGUMENT
 *   d_neighbors  int32[4n], d_residual uint32[4n], d_terminal int32[n]: the
 *                reduced graph on the device, updated in place as in
 *                gpupr_solve_reduced
 *   d_partition  uint8[n] device output, 1 = the node reaches the sink
 * The first call on a device looks up the array's device address (with that
 * device current) and caches it; make that first call before any stream
 * capture.  CUDA loads device modules lazily by default, so the array's
 * memory is committed when the module is first used: call
 * gpupr_noalloc_prepare() on each device before the caller's allocator
 * reserves the device heap (after a cudaDeviceReset, call it again: it looks
 * the address up anew).  Each call waits on the host for its stream (it reads
 * the solver's control block back between batches of steps) and returns
 * with the partition written.  It runs the one-launch-per-step engine (a
 * host check per 24 discharge rounds or 48 BFS levels), not the persistent
 * engine of gpupr_solve_reduced, so it is slower on the same graph; the
 * result is the same.  All calls share the one array and it keeps the last
 * call's contents (the call clears what must start at zero): calls whose
 * work overlaps on the GPU, from other streams or threads, race and corrupt
 * each other, so serialise them.
 */
gpupr_status gpupr_solve_reduced_noalloc(uint32_t n, int32_t* d_neighbors,
                                         uint32_t* d_residual, int32_t* d_terminal,
                                         uint8_t* d_partition,
                                         int32_t global_relabel_period,
                                         uint64_t max_rounds, int32_t local_steps,
                                         void* stream, gpupr_cut_stats* stats);

/*
 * Set-up of gpupr_solve_reduced_noalloc on the current device (no
 * counterpart in the reference): loads the solver's device module if CUDA has
 * not loaded it yet, which commits the static scratch array, and looks up the
 * array's device address anew.  Call it once per device before the caller's
 * allocator takes the device heap, and again after a cudaDeviceReset.
 * scratch_bytes (optional) receives the array's size.
 */
gpupr_status gpupr_noalloc_prepare(uint64_t* scratch_bytes);

/*
 * Topology upload (replaces wtivo.py:284-309, topology_to_cuda_chunked):
 * copies an Nx4 integer matrix from HOST memory (int32 or int64 elements,
 * elem_bytes 4 or 8; any byte strides, e.g. Fortran order) into a
 * contiguous int32 Nx4 device array d_out (16-byte aligned), narrowing int64
 * like numpy's astype(int32).  Returns once the host matrix has been read;
 * d_out is ready in the order of `stream`.
 */
gpupr_status gpupr_upload_topology(const void* host, uint64_t rows, int64_t row_stride_bytes,
                                   int64_t col_stride_bytes, int32_t elem_bytes, int32_t* d_out,
                                   void* stream);

/*
 * Edge-degree watertight audit (replaces is_watertight,
 * native/core/wtivo_core.cpp:402-464).  faces: n_faces x 3 int32 vertex ids,
 * in host memory or, with faces_on_device, device memory (e.g. the output of
 * gpupr_surface_fetch).  bad_groups = number of distinct undirected edges
 * whose face count is not 2 (the mesh is watertight when n_faces > 0 and
 * bad_groups == 0); table_bytes = device bytes of the edge table.  A
 * negative vertex id fails with GPUPR_ERR_INVALID_ARGUMENT, "negative vertex
 * index" (wtivo_core.cpp:424).
 */
gpupr_status gpupr_edge_audit(const int32_t* faces, uint64_t n_faces, int faces_on_device,
                              uint64_t* bad_groups, uint64_t* table_bytes, void* stream);

/*
 * Sparse unsigned distance grid, the input of the tet-centroid label sampler
 * (stands in for the reference's OpenVDB FloatGrid, native/vdb/wtivo_vdb.cpp:
 * 1007-1070, built with a linear transform of voxel_size): voxel (i,j,k)
 * sits at world (i,j,k) * voxel_size; bricks of 8^3 voxels; brick
 * (bx,by,bz) of a dims[0] x dims[1] x dims[2] box holds voxels
 * origin + 8*(bx,by,bz) + [0,8)^3.  table[(bx*dims[1] + by)*dims[2] + bz] is
 * the brick's number in values (-1: every voxel of it is the background);
 * values[brick*512 + (x*8 + y)*8 + z].  Voxels outside the box read the
 * background.  table/values live in device memory when on_device, else in
 * host memory (copied for the call).
 */
typedef struct {
    double voxel_size;
    int32_t origin[3];
    int32_t dims[3];
    float background;
    int32_t on_device;
    const int32_t* table;
    const float* values;
    uint64_t n_bricks;
} gpupr_brick_grid;

/*
 * Tet-centroid labels (replaces SparseUDF.sample_tet_labels,
 * native/vdb/wtivo_vdb.cpp:1519-1584): centroid = 0.25 * sum of the tet's 4
 * vertices, mapped to ((c - bbox_min)/(bbox_max - bbox_min))*(1 - 2 padding)
 * + padding, sampled with OpenVDB's BoxSampler semantics (trilinear over the
 * 8 voxels around floor(index), index = world / voxel_size); labels_out[i] =
 * 0 where the sample <= threshold, else 1.  tets (16-byte aligned when on the
 * device), vertices, labels_out and udf_out (optional: the samples) each in
 * host or device memory as flagged (udf_out follows labels_out).  Errors:
 * "SparseUDF.sample_tet_labels: degenerate bbox", "... tet index out of
 * range" (GPUPR_ERR_INVALID_ARGUMENT).
 */
gpupr_status gpupr_sample_tet_labels(const gpupr_brick_grid* grid, const double* vertices,
                                     uint64_t n_vertices, int vertices_on_device,
                                     const int32_t* tets, uint64_t n_tets, int tets_on_device,
                                     const double* bbox_min, const double* bbox_max,
                                     double padding, double threshold, uint8_t* labels_out,
                                     int labels_on_device, float* udf_out, void* stream);

/*
 * Autotuner (no counterpart in the reference).  The persistent engine's free
 * choices -- resident blocks per SM, the relabel work factor and chained
 * discharge -- change the time of a solve, never its result.  gpupr_autotune
 * builds the reduced graph of the given cut once, then times the solve
 * (restoring the graph each time), `reps` times each (default 3),
 * interleaved: first every pair of blocks per SM {1,2,3,4} and work factor
 * {0.25,0.5,1,2}, then, with the best pair, chaining off, 4 hops up to 4096 or
 * 32768 active nodes, 8 hops up to 131072, beside the built-in rule.  The
 * setting with the lowest median (the rule's own values when it wins) is
 * kept for the graph's size class (free nodes in [2^k, 2^(k+1))).  Later solves whose options leave those fields at 0 use
 * the table; classes without an entry keep the built-in size rule.  The
 * table is per process; gpupr_tune_table / gpupr_tune_table_set read and
 * replace it (to keep it across runs).  Arguments as gpupr_graph_cut.
 */
typedef struct {
    int32_t size_class;           /* k: free nodes in [2^k, 2^(k+1)) */
    int32_t blocks_per_sm;
    double work_relabel_factor;
    double solve_ms;              /* median solve time of the chosen setting */
    double default_ms;            /* median solve time under the built-in rule */
    int32_t chain_hops;           /* chained discharge (see gpupr_solve_options) */
    int32_t chain_max_active;
} gpupr_tune_entry;

gpupr_status gpupr_autotune(const double* vertices, uint64_t n_vertices, int vertices_on_device,
                            const int32_t* d_tets, const int32_t* d_neighbors, uint64_t n_tets,
                            const uint8_t* labels, int labels_on_device, double fill_T,
                            int32_t local_steps, int32_t reps, gpupr_tune_entry* chosen,
                            void* stream);
gpupr_status gpupr_tune_table(gpupr_tune_entry* entries, uint32_t capacity, uint32_t* count);
gpupr_status gpupr_tune_table_set(const gpupr_tune_entry* entries, uint32_t count);

/*
 * Batch autotuner (no counterpart in the reference): the same two stages as
 * gpupr_autotune on one batch (arguments as gpupr_graph_cut_batch), timing
 * the segmented solve of its union against the batch rule (the one
 * gpupr_graph_cut_batch applies when no entry exists).  The chosen setting is
 * kept in a separate per-process table keyed by the batch's size bucket: the
 * size class of its free nodes per graph (in [2^k, 2^(k+1))).  Later batches
 * whose options leave blocks_per_sm, work_relabel_factor, chain_hops and
 * chain_max_active at 0 take their bucket's entry.
 */
gpupr_status gpupr_autotune_batch(uint32_t n_graphs, const uint64_t* tet_offsets,
                                  const uint64_t* vertex_offsets, const double* vertices,
                                  int vertices_on_device, const int32_t* d_tets,
                                  const int32_t* d_neighbors, const uint8_t* labels,
                                  int labels_on_device, double fill_T, int32_t local_steps,
                                  int32_t reps, gpupr_tune_entry* chosen, void* stream);
gpupr_status gpupr_batch_tune_table(gpupr_tune_entry* entries, uint32_t capacity, uint32_t* count);
gpupr_status gpupr_batch_tune_table_set(const gpupr_tune_entry* entries, uint32_t count);

/* Release device memory cached between calls (pool + scratch). */
gpupr_status gpupr_release_cached_memory(void);

/* Bounded-wait self test: a device loop waits on a flag that nothing sets,
 * gives up after about `limit_us` microseconds and returns
 * GPUPR_ERR_TIMEOUT with the context still usable. */
gpupr_status gpupr_selftest_bounded_wait(uint32_t limit_us, void* stream);

#ifdef __cplusplus
}
#endif
#endif
