// gpupr_internal.cuh -- shared device structures and helpers of the B200
// graph-cut library.  Not part of the public ABI (include/wtivo_gpupr.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "wtivo_gpupr.h"

namespace gpupr {

// Unreached / unlabelled height.  Any height >= n (the free-node count) is
// inactive, exactly like the reference's source_h = n, inf_h = n + 1
// (gpu_push_relabel_fast.cu:426-427); UNVIS also marks "not visited" during
// a BFS, so no normalisation pass is needed (.cu:141-147 becomes a no-op).
constexpr uint32_t UNVIS = 0xFFFFFFFFu;

// Device control block: ring counters for the double-buffered queues, flags
// and work counters.  One per solve; zeroed at solve start.
struct Ctl {
    uint32_t act_cnt[3];     // active queue sizes, ring indexed by round % 3
    uint32_t bfs_cnt[3];     // BFS frontier sizes, ring indexed by level % 3
    uint32_t bfs_done;       // a level found an empty frontier
    uint32_t bfs_levels;     // levels expanded (non-empty) in this BFS
    int32_t error;           // first device invariant failure (status code)
    uint32_t error_node;
    uint32_t rounds_done;    // non-empty discharge rounds this phase
    uint32_t level_base;     // current BFS level (graph-launched batches)
    unsigned long long sink_flow;
    unsigned long long node_visits;
    unsigned long long pushes;
    unsigned long long bfs_visits;
    unsigned long long relabels;
    unsigned long long bar;  // persistent engine: barrier arrivals since launch
                             // (low 40 bits) | BAR_ABORT once an error is raised
    uint32_t relabel_phases; // persistent engine: global relabels run
    uint32_t pad0;
    // persistent engine, globaltimer ns of block 0 summed per phase: BFS
    // (seed + steps), active sweeps, discharge rounds
    unsigned long long bfs_ns, sweep_ns, discharge_ns;
    // segmented solves: graphs retired (no active node after an exact
    // relabel) and their free nodes
    unsigned long long retired_nodes;
    uint32_t segs_retired;
    // direction-optimizing relabels: the reached set the active sweep collects
    // for the next relabel, its size in the current relabel, nodes first
    // labelled per BFS step (ring by level, like bfs_cnt), sizes of the
    // bottom-up candidate lists (ring by bottom-up step), bottom-up steps run
    uint32_t cand_build;
    uint32_t cand_cnt;
    uint32_t lab_cnt[3];
    uint32_t bu_cnt[3];
    uint32_t bu_steps;
    // persistent engine: BFS steps by frontier size (<= 1024, <= 16384,
    // larger) and block 0's time in each class
    uint32_t step_cnt[3];
    uint32_t tail_L;         // persistent engine: BFS level after a tail step of block 0
    unsigned long long step_ns[3];
    unsigned long long tail_steps;   // tail steps and the levels they covered
    unsigned long long tail_levels;
    // tiled relabels: tile steps (grid barriers), tiles processed, nodes
    // loaded by them and labels they lowered
    unsigned long long tile_steps;
    unsigned long long tile_procs;
    unsigned long long tile_loads;
    unsigned long long tile_writes;
    // persistent engine: discharge rounds by active-set size (<= 4096,
    // <= 131072, larger) and block 0's time in each class
    uint32_t dround_cnt[3];
    unsigned long long dround_ns[3];
};

// Nodes per tile of a tiled relabel (a power of two; the persistent engine
// keeps one tile's labels and in-tile arcs in shared memory).
constexpr uint32_t RELABEL_TILE_SHIFT = 11;
constexpr uint32_t RELABEL_TILE = 1u << RELABEL_TILE_SHIFT;

// Nodes per pass of a whole-array sweep (seed, excess init, active sweep):
// 256 threads x 4 nodes.  Segmented solves keep the first graph of every such
// chunk.
constexpr uint32_t SWEEP_CHUNK = 1024u;

constexpr unsigned long long BAR_ABORT = 1ull << 62;
constexpr unsigned long long BAR_COUNT = (1ull << 40) - 1;

// View of the reduced graph + solver workspace handed to kernels.
struct SolveView {
    uint32_t n;
    const int4* __restrict__ nbr;       // [n] neighbor row (reduced ids, -1)
    uint32_t* res;                      // [4n] residual capacity per slot
    const uint8_t* __restrict__ rev;    // [n] 2-bit reverse slot per slot
    const uint4* __restrict__ pair;     // [n] per slot k: res[v][k] + res[u][rev k], the
                                        // arc pair's residual sum (u = nbr[v][k]); a push
                                        // moves residual between the two arcs and keeps it,
                                        // so r(u->v) = pair - res[v][k] between phases
    int4* inrow;                        // [n] persistent engine: per node the neighbours
                                        // with a residual arc into it (-1 elsewhere),
                                        // written by each relabel's seed sweep (null:
                                        // the BFS derives them from pair and res)
    uint8_t* inm;                       // [n] persistent engine, instead of inrow: bit k
                                        // = residual arc nbr[v][k] -> v, written by each
                                        // relabel's seed sweep from pair and res
    int32_t* term;                      // [n] src - snk residual
    long long* excess;                  // [n]
    uint32_t* height;                   // [n]
    uint32_t* act[2];                   // active queues (double buffered)
    uint32_t* fr[2];                    // BFS frontiers (fr[1] aliases act[1])
    Ctl* ctl;
    int local_steps;
    int chain_hops;                     // nodes one thread may discharge in a row in
                                        // one round (<= 1: no chaining) ...
    uint32_t chain_max_active;          // ... in rounds of at most this many nodes
    int bfs_block_levels;               // persistent engine: > 1 = BFS steps expand that many
                                        // levels per block from its shared stage (0: chains)
    int bfs_hops;                       // nodes one thread may label in a row in one
                                        // short BFS step (<= 1: level by level)
    // Segmented solve (a batch: independent graphs, each a contiguous node
    // range; persistent engine).  nseg == 0: one graph.
    uint32_t nseg;
    const uint32_t* __restrict__ seg_off;    // [nseg+1] first node of each graph
    const uint32_t* __restrict__ chunk_seg;  // [ceil(n/SWEEP_CHUNK)] first graph of each chunk
    uint32_t* seg_live;                 // [nseg] nonzero while the graph is being solved
    uint32_t* seg_act;                  // [nseg] the last active sweep found an active node
    // Direction-optimizing relabels (persistent engine): candidate lists of
    // n entries each, and the switch ratio (bottom_up == 0: top-down only)
    uint32_t* cand[2];
    int bottom_up;
    float bu_ratio;
    uint32_t bfs_chain_max;             // BFS steps chain (bfs_hops) over frontiers up to this size
    int warp_agg;                       // discharge: lanes pushing to the same neighbour
                                        // share one excess atomic
    uint32_t tail_max;                  // persistent engine: frontiers up to this size are
                                        // expanded by block 0 alone, level after level
                                        // (0: never)
    // Tiled relabels (persistent engine; arcm == null: frontier steps).  The
    // nodes are cut into tiles of RELABEL_TILE consecutive ids; a relabel
    // solves the BFS inside each tile in shared memory and re-queues a tile
    // only when a label its nodes read from another tile went down.
    uint8_t* arcm;                      // [n] per node: bit k = residual arc to neighbour k,
                                        // bit 4+k = residual arc from it (seed sweep)
    uint32_t* tile_stamp;               // [ntiles] last tile step the tile was queued for
    uint32_t ntiles;
};

// ---------------------------------------------------------------------------
// Host-side helpers
// ---------------------------------------------------------------------------
struct Error {
    gpupr_status status;
    std::string msg;
};

void set_last_error(const std::string& msg);

#define GPUPR_CUDA(expr)                                                     \
    do {                                                                     \
        cudaError_t _e = (expr);                                             \
        if (_e != cudaSuccess)                                               \
            throw ::gpupr::Error{_e == cudaErrorMemoryAllocation             \
                                     ? GPUPR_ERR_OUT_OF_MEMORY               \
                                     : GPUPR_ERR_CUDA,                       \
                                 std::string("GPUPr-B200 CUDA failure at ") + \
                                     #expr + ": " + cudaGetErrorString(_e)}; \
    } while (0)

// Stream-ordered device allocation from the library's pool.
void* pool_alloc(size_t bytes, cudaStream_t s);
void pool_free(void* p, cudaStream_t s);

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t st) : n(count), s(st)
    {
        if (count) p = static_cast<T*>(pool_alloc(count * sizeof(T), st));
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) { reset(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p) pool_free(p, s);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Copies between pageable host arrays and the device through pinned staging
// and a host copy pool (hostio.cu).  host_to_device returns once the host
// array has been read (the device copy is ordered on s); device_to_host
// returns once the host array holds the data.
void host_to_device(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s);
void device_to_host(void* h_dst, const void* d_src, size_t bytes, cudaStream_t s);
void upload_topology(int32_t* d_out, const void* host, uint64_t rows, int64_t row_stride,
                     int64_t col_stride, int elem_bytes, cudaStream_t s);

// Per-thread cached host resources of the current device (hostio.cu): a
// pinned mirror of the solver control block and timing events (slots 0-7;
// 0-1 build timer, 2-5 solver).  A call creates and frees none of them, so
// it never pays for pinning host pages, nor for the device-wide
// synchronisation that freeing pinned memory implies.
Ctl* pinned_ctl();
cudaEvent_t timing_event(int slot);

// Launch geometry: number of SMs of the current device (cached).
int sm_count();

// ---------------------------------------------------------------------------
// Reduced-graph build (graph_build.cu)
// ---------------------------------------------------------------------------
struct BuildInputs {
    const double* d_vertices;   // device [nv*3]
    uint64_t nv;
    const int32_t* d_tets;      // device [N*4]
    const int32_t* d_nbrs;      // device [N*4]
    const uint8_t* d_labels;    // device [N]
    uint64_t N;
    double fill_T;
    bool want_base_node = false;       // also keep min(src, snk) per free node
};

struct BuildInfo {
    uint64_t free_n = 0, fixed_source = 0, fixed_sink = 0, full_refs = 0;
    uint64_t free_refs = 0, terminal_edges = 0;
    int64_t terminal_base_flow = 0;
};

struct ReducedGraph {
    uint32_t n = 0;
    DevBuf<int4> nbr;
    DevBuf<uint32_t> res;       // 4n
    DevBuf<uint8_t> rev;
    DevBuf<uint32_t> pair;      // 4n: cap(u->v) + cap(v->u) per slot
    DevBuf<int32_t> term;
    DevBuf<int32_t> full_to_free;  // N
    DevBuf<uint32_t> free_old;     // n
    DevBuf<uint32_t> base_node;    // n, only when BuildInputs::want_base_node
    uint64_t graph_bytes() const
    {
        return nbr.bytes() + res.bytes() + rev.bytes() + pair.bytes() + term.bytes();
    }
};

// Classify + compact + build; throws gpupr::Error with reference messages.
void build_reduced_graph(const BuildInputs& in, ReducedGraph& g, BuildInfo& info,
                         cudaStream_t s, uint64_t* launches);

// Batches (batch.cu): G graphs packed end to end.  Local vertex/neighbor ids
// become global ids; per-graph sums run over contiguous ranges.
void batch_pack(uint64_t N, uint32_t G, const unsigned long long* d_tet_off,
                const unsigned long long* d_vert_off, const int32_t* d_tets_local,
                const int32_t* d_nbrs_local, int32_t* d_tets, int32_t* d_nbrs, cudaStream_t s,
                uint64_t* launches);
void batch_free_counts(uint32_t G, const unsigned long long* d_tet_off, const int32_t* d_full_to_free,
                       unsigned long long* d_counts, cudaStream_t s, uint64_t* launches);
void batch_flows(uint32_t G, const unsigned long long* d_free_off, const int32_t* d_term,
                 const long long* d_excess, const uint32_t* d_base_node, long long* d_raw,
                 unsigned long long* d_base, cudaStream_t s, uint64_t* launches);

// Exclusive scan of per-tile counts (one block); *d_total receives the sum.
void scan_tile_counts(uint32_t ntiles, const uint32_t* d_cnt, unsigned long long* d_off,
                      unsigned long long* d_total, cudaStream_t s, uint64_t* launches);

// Reverse-slot table and arc-pair residual sums (pair[v][k] = res[v][k] +
// res[u][rev k]) of a reduced graph given in the reference layout, from its
// current residuals.
void compute_reverse_slots(uint32_t n, const int4* d_nbr, const uint32_t* d_res, uint8_t* d_rev,
                           uint32_t* d_pair, cudaStream_t s, uint64_t* launches);

// label scatter: out[free_old[q]] = height[q] != UNVIS
void scatter_partition(uint32_t n, const uint32_t* d_free_old, const uint32_t* d_height,
                       uint8_t* d_out, cudaStream_t s, uint64_t* launches);
void partition_from_height(uint32_t n, const uint32_t* d_height, uint8_t* d_part,
                           cudaStream_t s, uint64_t* launches);

// ---------------------------------------------------------------------------
// Solver (push_relabel.cu)
// ---------------------------------------------------------------------------
struct SolveOptions {
    int local_steps = 8;
    int relabel_rounds = 128;      // ceil(period / local_steps), 0 = only when idle
    int period = 1024;             // global_relabel_period as given (clamped, 0 = none)
    uint64_t max_rounds = 2000000ull;
    double time_limit_s = 240.0;
    int round_batch = 24;
    int bfs_batch = 48;
    int block = 256;
    int blocks_per_sm = 0;         // 0: by graph size (persistent), 4 (one launch per step)
    double work_factor = 0.0;      // node visits per node between relabels, 0 = engine default
    int engine = 0;                // 0 auto, 1 one launch per step, 2 persistent
    int chain_hops = 0;            // persistent engine: 0 = default
    int chain_max_active = 0;      // persistent engine: 0 = default
    int bfs_chain_hops = 0;        // persistent engine: 0 = default
    int bfs_tail_max = 0;          // persistent engine: 0 = default, < 0 = never
    int discharge_warp_aggregate = 0;   // persistent engine: 1 = warp-aggregated excess atomics
    int bfs_chain_max_frontier = 0;     // persistent engine: 0 = default (no limit)
    int bfs_bottom_up = 0;         // persistent engine: direction-optimizing relabels
    double bfs_bottom_up_ratio = 1.0;
    int max_blocks_per_sm = 0;     // persistent engine: cap on the grid (0 = none); the
                                   // server's lanes use it so their solves fit side by side
    int relabel_tiles = 0;         // persistent engine: 1 = tiled relabels, < 0 = frontier
                                   // steps, 0 = default
    int bfs_block_levels = 0;      // persistent engine: > 1 = block sub-levels per BFS step
    int bfs_in_arc_masks = 0;      // persistent engine: 1 = in-arc masks, < 0 = in-arc rows,
                                   // 0 = default
};

SolveOptions resolve_options(const gpupr_solve_options* o, int local_steps_raw,
                             int period_raw, uint64_t max_rounds_raw);

struct SolveWorkspace {
    DevBuf<long long> excess;
    DevBuf<uint32_t> height;
    DevBuf<uint32_t> q0, q1, q2;
    DevBuf<Ctl> ctl;
    DevBuf<uint32_t> chunk_seg, seg_live, seg_act;   // segmented solves only
    DevBuf<uint32_t> cand0, cand1;                   // direction-optimizing relabels only
    DevBuf<int4> inrow;                              // persistent engine: in-arc rows
    DevBuf<uint8_t> inm;                             // persistent engine: in-arc masks
    DevBuf<uint8_t> arcm;                            // tiled relabels: arc masks
    DevBuf<uint32_t> tile_stamp;                     // tiled relabels: queue stamps
    uint64_t bytes() const
    {
        return excess.bytes() + height.bytes() + q0.bytes() + q1.bytes() + q2.bytes() + ctl.bytes() +
               chunk_seg.bytes() + seg_live.bytes() + seg_act.bytes() + cand0.bytes() + cand1.bytes() +
               inrow.bytes() + inm.bytes() + arcm.bytes() + tile_stamp.bytes();
    }
};

// The graphs of a batch as node ranges of the reduced union graph: graph k
// owns reduced ids [d_off[k], d_off[k+1]) (device, nseg + 1 entries).
struct Segments {
    uint32_t nseg = 0;
    const uint32_t* d_off = nullptr;
};

struct SolveResult {
    int64_t raw_flow = 0;
    uint64_t rounds = 0, relabels = 0, node_visits = 0, pushes = 0, bfs_visits = 0,
             bfs_levels = 0, launches = 0;
    double solve_s = 0.0, final_relabel_s = 0.0, solve_device_ms = 0.0;
    double discharge_ms = 0.0, bfs_ms = 0.0, sweep_ms = 0.0;
    uint64_t discharge_launches = 0, bfs_launches = 0;
    uint64_t workspace_bytes = 0;
    uint64_t graphs_retired = 0;   // segmented solves: graphs finished before the last relabel
    uint64_t bottom_up_steps = 0;  // BFS steps run bottom-up
    uint64_t tail_steps = 0, tail_levels = 0;   // BFS tail steps of block 0, levels covered
    uint64_t step_cnt[3] = {0, 0, 0};  // BFS steps by frontier size (<= 1024, <= 16384, larger)
    double step_ms[3] = {0, 0, 0};
    int engine = 1;                // 1 one launch per step, 2 persistent
    int blocks_per_sm = 0;         // persistent engine: grid used
    double work_factor = 0.0;      // persistent engine: relabel work factor used
    int chain_hops = 0, chain_max_active = 0;   // persistent engine: chaining used
    int relabel_tiles = 0;         // persistent engine: 1 = tiled relabels ran
    uint64_t tile_steps = 0, tile_procs = 0, tile_loads = 0, tile_writes = 0;
    uint64_t dround_cnt[3] = {0, 0, 0};  // discharge rounds by active nodes (<= 4096, <= 131072, larger)
    double dround_ms[3] = {0, 0, 0};
};

// Autotuner table (push_relabel.cu): per size class (floor(log2 n)), the
// persistent engine's blocks per SM and relabel work factor.
struct TuneEntry {
    int32_t size_class = 0, blocks_per_sm = 0;
    double work_factor = 0.0, solve_ms = 0.0, default_ms = 0.0;
    int32_t chain_hops = 4, chain_max_active = 4096;
};
bool tune_lookup(uint32_t n, TuneEntry* out);
void tune_store(const TuneEntry& e);
std::vector<TuneEntry> tune_all();
void tune_replace(const std::vector<TuneEntry>& entries);
int size_class(uint32_t n);
// The batch table, by the size class of the free nodes per graph.
bool batch_tune_lookup(uint64_t mean_free, TuneEntry* out);
void batch_tune_store(const TuneEntry& e);
std::vector<TuneEntry> batch_tune_all();
void batch_tune_replace(const std::vector<TuneEntry>& entries);

// Phase-I push-relabel on a reduced graph (res/term updated in place).
// On return the workspace heights mark the sink-reachable set
// (height != UNVIS) of the final residual graph.
// With segments (a batch), the persistent engine retires each graph once an
// exact relabel finds no active node in it; the one-launch-per-step engine
// solves the union as one graph.
void solve_push_relabel(uint32_t n, const int4* d_nbr, uint32_t* d_res, const uint8_t* d_rev,
                        const uint32_t* d_pair, int32_t* d_term, SolveWorkspace& w,
                        const SolveOptions& opt, cudaStream_t s, SolveResult& out,
                        const Segments* segments = nullptr);

// Cut-surface extraction (surface.cu): count keeps its result per thread
// for the following fetch.
void surface_count(const uint8_t* labels, int l_dev, const double* vertices, uint64_t nv, int v_dev,
                   const int32_t* d_tets, const int32_t* d_nbrs, uint64_t N, uint64_t* n_faces,
                   uint64_t* n_used, cudaStream_t s);
void surface_fetch(int32_t* faces, double* verts, int out_dev, cudaStream_t s);

// Sparse unsigned distance grid of 8^3-voxel bricks in device memory (the
// layout of gpupr_brick_grid) and the tet-centroid label sampler
// (labels.cu): labels[i] = 0 where the box-sampled distance at tet i's
// centroid is <= threshold, else 1; udf (optional) receives the samples.
struct BrickGridDesc {
    double voxel_size;
    int32_t origin[3];
    int32_t dims[3];
    float background;
    const int32_t* d_table;
    const float* d_values;
};

void sample_tet_labels(const BrickGridDesc& grid, const double* d_vertices, uint64_t nv,
                       const int32_t* d_tets, uint64_t nt, const double* bmin, const double* bmax,
                       double padding, double threshold, uint8_t* d_labels, float* d_udf,
                       cudaStream_t s, uint64_t* launches);

// Edge-degree watertight audit of F device faces (audit.cu): the number of
// distinct undirected edges whose face count is not 2, and the bytes of the
// device edge table used.
void edge_audit(const int32_t* d_faces, uint64_t nf, cudaStream_t s, uint64_t* bad_groups,
                uint64_t* table_bytes, uint64_t* launches);

// Allocation-free solve (push_relabel.cu): all scratch in a static device
// array sized for NOALLOC_MAX_NODES nodes; the partition goes to d_partition.
constexpr uint32_t NOALLOC_MAX_NODES = 1u << 20;
void solve_reduced_noalloc(uint32_t n, int32_t* d_nbr, uint32_t* d_res, int32_t* d_term,
                           uint8_t* d_partition, const SolveOptions& opt, cudaStream_t s,
                           SolveResult& out);
// Looks up (again) the static scratch array's device address on the current
// device, loading its module if needed; returns the array's size in bytes.
uint64_t noalloc_prepare();
void compute_reverse_slots_noalloc(uint32_t n, const int4* d_nbr, const uint32_t* d_res,
                                   uint8_t* d_rev, uint32_t* d_pair, int32_t* d_err,
                                   cudaStream_t s);

// Batched graph cut (capi.cu), used by the C ABI and the serving loop;
// max_blocks_per_sm caps the persistent solve's grid (0 = no cap).
void run_graph_cut_batch(uint32_t G, const uint64_t* toff, const uint64_t* voff,
                         const double* vertices, int v_dev, const int32_t* d_tets_l,
                         const int32_t* d_nbrs_l, const uint8_t* labels, int l_dev, double fill_T,
                         const gpupr_solve_options* options, uint8_t* out, int out_dev,
                         cudaStream_t s, gpupr_batch_item* items, gpupr_cut_stats* st,
                         int max_blocks_per_sm = 0);

// Resident blocks per SM of the persistent solver kernel on the current
// device (its occupancy limit).
int persistent_blocks_per_sm();

// Bounded wait self test kernel driver.
gpupr_status bounded_wait_selftest(uint32_t limit_us, cudaStream_t s);

// Raw ELL graph: res = cap, term = src - snk, returns base flow sum min(src,snk).
int64_t prepare_raw_graph(uint32_t n, const uint32_t* d_cap, const uint32_t* d_src,
                          const uint32_t* d_snk, const int32_t* d_nbr, uint32_t* d_res,
                          int32_t* d_term, cudaStream_t s, uint64_t* launches);

}  // namespace gpupr
