// push_relabel.cu -- Phase-I multi-discharge push-relabel on the reduced
// ELL graph, with global relabels by backward BFS from the sink.
//
// Replaces cellocut_gpu_push_relabel_fast
// (native/gpupr/gpu_push_relabel_fast.cu:406-571).  Differences in design:
//
//  * No host round trip per round or per BFS level.  The default engine is
//    one persistent cooperative kernel (k_solve_persistent) that runs the
//    whole solve, steps separated by a bounded software grid barrier; the
//    other engine launches one kernel per step, reading queue sizes from a
//    device control block (ring counters), with the host checking the state
//    once per batch of steps.
//  * Chained discharge: the thread that takes ownership of a neighbour's
//    excess may discharge it at once, so excess moves several hops a round.
//  * Label-correcting BFS steps (persistent engine): labels are lowered by
//    atomicMin, and after expanding its share of the frontier each block
//    expands the nodes it labelled itself for up to 16 levels from its
//    shared-memory stage (or, as an option, a thread labels several nodes in
//    a row), so one grid barrier covers several levels; reachability is
//    exact in every case and labels converge to distances while lowered
//    labels propagate.  The active queue is collected after each BFS by a
//    streaming sweep, in node order (engine 1 appends it during its
//    level-synchronous BFS, .cu:360-402 and :149-166).
//  * Reverse slots are precomputed at build time (2 bits per slot), so a push
//    never searches the neighbor's row (.cu:56-67).
//  * The backward BFS reads no residual of the neighbour it labels: each arc
//    pair keeps the sum of its two residuals (pushes move residual between
//    the two arcs and never change the sum), so r(v->u) = pair[u][k] -
//    res[u][k] comes from the frontier node u's own rows (.cu:103-139 read
//    the neighbour's row and searched it for the reverse slot).
//  * Queue de-duplication without flags: a node owns its excess; the thread
//    whose atomic add moves a node's excess from 0 to positive enqueues it,
//    and a discharged node that keeps excess re-enqueues itself (.cu:168-178
//    used a queued[] flag and a CAS per enqueue).
//  * Queue appends are staged in shared memory and written with one global
//    atomic per block iteration; sink flow and work counters are reduced per
//    block.
//  * As an option, relabels by tiles of consecutive nodes: each tile's BFS
//    runs in shared memory and a tile is re-run only when a label it reads
//    from another tile goes down (exact distances at the fixpoint).
//  * Exactness by construction: the solve ends only when a global relabel
//    (reachability exact) finds no node with excess that can reach the sink, so the
//    returned preflow is maximum and the sink-reachable set is the minimal
//    sink side of the minimum cut (the reference stops when its queue
//    empties, .cu:490, then relabels once, .cu:551-556).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <cmath>
#include <string>

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "gpupr_internal.cuh"

namespace cg = cooperative_groups;

namespace gpupr {
namespace {

constexpr int DTPB = 256;   // block size of the solver kernels

__device__ __forceinline__ uint32_t ldcg(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ int32_t ldcg(const int32_t* p) { return __ldcg(p); }
__device__ __forceinline__ long long ldcg(const long long* p) { return __ldcg(p); }

// A load that bypasses the caches' stale copies (control counters written by
// other blocks before the last grid barrier).
template <class T>
__device__ __forceinline__ T vload(const T* p) { return *reinterpret_cast<const volatile T*>(p); }

template <class T>
__device__ __forceinline__ T warp_block_sum(T v, T* sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x < 32) {
        t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : T(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;
}

// Records the first device error and makes every block waiting in (or later
// reaching) a grid barrier of the persistent engine leave it.
__device__ __forceinline__ void raise_error(Ctl* ctl, int code)
{
    atomicCAS(&ctl->error, 0, code);
    atomicOr(&ctl->bar, BAR_ABORT);
}

// Copy a block's staged entries to a global queue of capacity cap.  Queue
// entries are unique by construction (each node is appended at most once per
// round or BFS); the guard keeps the writes inside the buffer even if that
// invariant were broken, and reports it instead.
__device__ __forceinline__ void flush_stage(const uint32_t* s_src, uint32_t count, uint32_t base,
                                            uint32_t* dst, uint32_t cap, Ctl* ctl)
{
    if (threadIdx.x == 0 && (uint64_t)base + count > cap) raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
    for (uint32_t j = threadIdx.x; j < count; j += DTPB)
        if (base + j < cap) dst[base + j] = s_src[j];
}

__global__ void __launch_bounds__(DTPB) k_init_excess(uint32_t n, const int32_t* __restrict__ term,
                                                      long long* __restrict__ excess)
{
    for (uint32_t v = blockIdx.x * DTPB + threadIdx.x; v < n; v += gridDim.x * DTPB) {
        const int32_t t = term[v];
        excess[v] = t > 0 ? (long long)t : 0ll;   // source arc saturated (.cu:69-83)
    }
}

// Frontier size up to which a BFS level of the one-launch-per-step engine
// loads the excess of every neighbour with an arc into the frontier node at
// once (above it, only the excess of a node it labels).
constexpr uint32_t BFS_EAGER_MAX = 32768u;

// Nodes per thread in the whole-array passes (BFS seed, excess init): that
// many independent loads in flight per thread make the pass stream instead
// of waiting for one round trip per node.
constexpr int SWEEP_UNROLL = 4;
static_assert(DTPB * SWEEP_UNROLL == (int)SWEEP_CHUNK, "sweep chunk of the segment table");

// The graph of node v in a segmented solve, searched forward from seg (the
// first graph of v's sweep chunk; graphs without nodes are stepped over).
__device__ __forceinline__ uint32_t seg_of(const SolveView& g, uint32_t seg, uint32_t v)
{
    while (seg + 1u < g.nseg && __ldg(g.seg_off + seg + 1u) <= v) ++seg;
    return seg;
}

// Whether a sweep handles node v: every node of a single graph; in a
// segmented solve only nodes of graphs not yet retired.  *seg: v's graph.
__device__ __forceinline__ bool sweep_node(const SolveView& g, uint32_t seg0, uint32_t v, uint32_t* seg)
{
    *seg = 0u;
    if (v >= g.n) return false;
    if (!g.nseg) return true;
    *seg = seg_of(g, seg0, v);
    return ldcg(g.seg_live + *seg) != 0u;
}

// The neighbours v of node u with a residual arc v -> u, as a row (-1 where
// there is none): r(v->u) = pair[u][k] - res[u][k], exact between phases.
__device__ __forceinline__ int4 in_arc_row(const SolveView& g, uint32_t u)
{
    const int4 nb4 = __ldg(g.nbr + u);
    const uint4 p4 = __ldg(g.pair + u);
    const uint4 r4 = __ldcg(reinterpret_cast<const uint4*>(g.res) + u);
    return make_int4(p4.x > r4.x ? nb4.x : -1, p4.y > r4.y ? nb4.y : -1, p4.z > r4.z ? nb4.z : -1,
                     p4.w > r4.w ? nb4.w : -1);
}

// The same in-arcs as a mask (bit k: residual arc nbr[v][k] -> v), from v's
// pair sums and residuals alone: a slot without a neighbour has pair sum 0.
__device__ __forceinline__ uint32_t in_arc_mask(const SolveView& g, uint32_t v)
{
    const uint4 p4 = __ldg(g.pair + v);
    const uint4 r4 = __ldcg(reinterpret_cast<const uint4*>(g.res) + v);
    return (uint32_t)(p4.x > r4.x) | ((uint32_t)(p4.y > r4.y) << 1) | ((uint32_t)(p4.z > r4.z) << 2) |
           ((uint32_t)(p4.w > r4.w) << 3);
}

// A node's arc mask for a tiled relabel: bit k = residual arc v -> nbr[v][k]
// (res > 0), bit 4+k = residual arc nbr[v][k] -> v (pair - res > 0), both
// exact between phases.
__device__ __forceinline__ uint32_t arc_mask(const SolveView& g, uint32_t v)
{
    const int4 nb4 = __ldg(g.nbr + v);
    const uint4 p4 = __ldg(g.pair + v);
    const uint4 r4 = __ldcg(reinterpret_cast<const uint4*>(g.res) + v);
    const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
    const uint32_t r[4] = {r4.x, r4.y, r4.z, r4.w}, pr[4] = {p4.x, p4.y, p4.z, p4.w};
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (nb[k] < 0) continue;
        m |= (uint32_t)(r[k] > 0u) << k;
        m |= (uint32_t)(pr[k] > r[k]) << (4 + k);
    }
    return m;
}

// Queues tile t for tile step `step` unless it is queued for it already (the
// stamp holds the last step a tile was queued for; steps only grow within a
// solve, so each tile enters a step's queue at most once and the queue,
// RELABEL_TILE-fold shorter than a node queue, cannot overflow).
__device__ __forceinline__ void queue_tile(const SolveView& g, uint32_t t, uint32_t step)
{
    if (atomicMax(g.tile_stamp + t, step) >= step) return;
    uint32_t* q = (step & 1u) ? g.fr[1] : g.fr[0];
    const uint32_t pos = atomicAdd(&g.ctl->bfs_cnt[step % 3u], 1u);
    if (pos < g.ntiles) q[pos] = t;
    else raise_error(g.ctl, (int)GPUPR_ERR_INVARIANT);
}

// Level 1 of the backward BFS: nodes with a residual arc to the sink.  Every
// other height is reset to UNVIS (.cu:374-379).  With g.inm (persistent
// engine, default) the same streaming pass writes every node's in-arc mask,
// with g.inrow its in-arc row, so a BFS step reads the frontier node's
// neighbour row and mask byte, or its in-arc row, instead of three rows.  s_m[0..5] are the block's
// staging counters (frontier count, active count, and their flush copies);
// s_fr and s_act hold DTPB * SWEEP_UNROLL entries each.  With kActive the
// seeds that hold excess are appended to the active queue (engine 1; the
// persistent engine finds the active nodes after the BFS, active_sweep_body).
// With g.arcm (tiled relabels) the pass writes every node's arc mask instead
// of an in-arc row and queues the tiles holding a seed for tile step
// `tile_step`; the seeds are not appended to a frontier.
template <bool kActive>
__device__ __forceinline__ void bfs_seed_body(const SolveView& g, uint32_t* s_fr, uint32_t* s_act,
                                              uint32_t* s_m, uint32_t tile_step = 0u)
{
    Ctl* ctl = g.ctl;
    constexpr uint32_t CH = DTPB * SWEEP_UNROLL;
    for (uint32_t base = blockIdx.x * CH; base < g.n; base += gridDim.x * CH) {
        const uint32_t seg0 = g.nseg ? __ldg(g.chunk_seg + base / CH) : 0u;
        bool in[SWEEP_UNROLL];
        int32_t t[SWEEP_UNROLL];
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            uint32_t sg;
            in[j] = sweep_node(g, seg0, v, &sg);   // a retired graph keeps its labels
            t[j] = in[j] ? ldcg(g.term + v) : 0;
        }
        long long x[SWEEP_UNROLL];
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            x[j] = (kActive && in[j] && t[j] < 0) ? ldcg(g.excess + v) : 0ll;
            if (in[j]) g.height[v] = (t[j] < 0) ? 1u : UNVIS;
        }
        if (g.arcm) {
            // a warp's 32 nodes lie in one tile (RELABEL_TILE is a multiple of 32)
#pragma unroll
            for (int j = 0; j < SWEEP_UNROLL; ++j) {
                const uint32_t v = base + j * DTPB + threadIdx.x;
                if (in[j]) g.arcm[v] = (uint8_t)arc_mask(g, v);
                const unsigned seeds = __ballot_sync(0xffffffffu, in[j] && t[j] < 0);
                if (seeds && (int)(threadIdx.x & 31u) == __ffs(seeds) - 1)
                    queue_tile(g, v >> RELABEL_TILE_SHIFT, tile_step);
            }
            continue;   // no frontier: the tile steps start from the queued tiles
        }
        if (g.inm) {
#pragma unroll
            for (int j = 0; j < SWEEP_UNROLL; ++j) {
                const uint32_t v = base + j * DTPB + threadIdx.x;
                if (in[j]) g.inm[v] = (uint8_t)in_arc_mask(g, v);
            }
        } else if (g.inrow) {
#pragma unroll 2
            for (int j = 0; j < SWEEP_UNROLL; ++j) {
                const uint32_t v = base + j * DTPB + threadIdx.x;
                if (in[j]) __stcg(g.inrow + v, in_arc_row(g, v));
            }
        }
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            if (in[j] && t[j] < 0) {
                s_fr[atomicAdd(&s_m[0], 1u)] = v;
                if (kActive && 1u < g.n && x[j] > 0) s_act[atomicAdd(&s_m[1], 1u)] = v;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[2] = s_m[0]; s_m[3] = s_m[1]; s_m[0] = 0; s_m[1] = 0;
            s_m[4] = s_m[2] ? atomicAdd(&ctl->bfs_cnt[1], s_m[2]) : 0u;
            s_m[5] = s_m[3] ? atomicAdd(&ctl->act_cnt[0], s_m[3]) : 0u;
            if (g.bottom_up && s_m[2]) atomicAdd(&ctl->lab_cnt[1], s_m[2]);
        }
        __syncthreads();
        flush_stage(s_fr, s_m[2], s_m[4], g.fr[1], g.n, ctl);
        flush_stage(s_act, s_m[3], s_m[5], g.act[0], g.n, ctl);
        __syncthreads();
    }
}

// Nodes one thread may label in a row in a short BFS step (bfs_step_body).
constexpr int BFS_CHAIN_HOPS = 4;

// Queues up to this size are spread over every SM (queue_index).
constexpr uint32_t SPREAD_MAX = 65536u;

// Queue index of a thread's entry in pass `it` over a queue of cnt entries;
// pass `it` covers indices [it * gridDim.x * DTPB, (it + 1) * gridDim.x * DTPB).
// A short queue (cnt <= SPREAD_MAX) is dealt to warps in 32-entry chunks
// round-robin over the blocks, so it is spread over every SM; measured on
// B200, a BFS level of 2-4K nodes on the first 8-16 blocks (12 random loads
// per node in flight, thousands per SM) took ~9.7 us, spread ~7.5 us.  A long
// queue keeps 256 consecutive entries per block: they were appended by one
// block of the step before and are near each other in the graph, and the
// spread order made levels of 262K+ nodes 15% slower.
__device__ __forceinline__ uint32_t queue_index(uint32_t it, uint32_t cnt)
{
    if (cnt <= SPREAD_MAX) {
        const uint32_t chunk = (it * (DTPB / 32) + (threadIdx.x >> 5)) * gridDim.x + blockIdx.x;
        return chunk * 32u + (threadIdx.x & 31u);
    }
    return (it * gridDim.x + blockIdx.x) * DTPB + threadIdx.x;
}

// The active queue after a BFS of the persistent engine: every node with a
// label below n and positive excess, appended in node order by one streaming
// pass (12 bytes a node) instead of a random excess load for each node the
// BFS labels.  s_act holds DTPB * SWEEP_UNROLL entries; s_m[1], s_m[3] and
// s_m[5] are its staging counters.  In a segmented solve it also marks the
// graphs that still hold an active node.  With direction-optimizing relabels
// the same pass collects every reached node (label below UNVIS) into
// cand[0], staged in s_cand (DTPB * SWEEP_UNROLL entries, counters
// s_m[7..9]): the candidates of the next relabel's bottom-up steps.
__device__ __forceinline__ void active_sweep_body(const SolveView& g, uint32_t* s_act, uint32_t* s_cand,
                                                  uint32_t* s_m)
{
    Ctl* ctl = g.ctl;
    constexpr uint32_t CH = DTPB * SWEEP_UNROLL;
    for (uint32_t base = blockIdx.x * CH; base < g.n; base += gridDim.x * CH) {
        const uint32_t seg0 = g.nseg ? __ldg(g.chunk_seg + base / CH) : 0u;
        uint32_t h[SWEEP_UNROLL], sg[SWEEP_UNROLL];
        long long x[SWEEP_UNROLL];
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            const bool in = sweep_node(g, seg0, v, &sg[j]);
            h[j] = in ? ldcg(g.height + v) : UNVIS;
            x[j] = in ? ldcg(g.excess + v) : 0ll;
        }
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const bool act = h[j] < g.n && x[j] > 0;
            if (act) s_act[atomicAdd(&s_m[1], 1u)] = base + j * DTPB + threadIdx.x;
            if (g.bottom_up && h[j] != UNVIS) s_cand[atomicAdd(&s_m[7], 1u)] = base + j * DTPB + threadIdx.x;
            if (g.nseg) {
                // the graph still has work: one store per group of lanes in the same graph
                const unsigned grp = __match_any_sync(0xffffffffu, act ? sg[j] : 0xFFFFFFFFu);
                if (act && (int)(threadIdx.x & 31u) == __ffs(grp) - 1) g.seg_act[sg[j]] = 1u;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[3] = s_m[1]; s_m[1] = 0;
            s_m[5] = s_m[3] ? atomicAdd(&ctl->act_cnt[0], s_m[3]) : 0u;
            s_m[8] = s_m[7]; s_m[7] = 0;
            s_m[9] = s_m[8] ? atomicAdd(&ctl->cand_build, s_m[8]) : 0u;
        }
        __syncthreads();
        flush_stage(s_act, s_m[3], s_m[5], g.act[0], g.n, ctl);
        if (g.bottom_up) flush_stage(s_cand, s_m[8], s_m[9], g.cand[0], g.n, ctl);
        __syncthreads();
    }
}

// A thread's first entry of a short queue (queue_index(0, cnt <= SPREAD_MAX)),
// loaded by an L2 load that stays in program order before the queue-size read
// that follows it, so the two round trips overlap.  Entries at or past the
// queue size are stale and are never used; the queues hold n entries.
__device__ __forceinline__ uint32_t prefetch_entry(const uint32_t* in, uint32_t n)
{
    const uint32_t i = queue_index(0, 0u);
    uint32_t v = 0;
    if (i < n) asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(in + i) : "memory");
    return v;
}

// The neighbours v of frontier node u with a residual arc v -> u, from u's
// own rows: r(v->u) = pair[u][k] - res[u][k] (exact between phases, when no
// push is in flight).  Returns u's neighbour row; bit k of *arcs is slot k.
__device__ __forceinline__ int4 in_arcs_written(const SolveView& g, uint32_t u)
{
    // what this relabel's seed sweep wrote (L2 loads: other blocks wrote it):
    // u's in-arc row, or its neighbour row masked by its in-arc mask
    if (!g.inm) return __ldcg(g.inrow + u);
    const int4 nb4 = __ldg(g.nbr + u);
    const uint32_t m = __ldcg(g.inm + u);
    return make_int4((m & 1u) ? nb4.x : -1, (m & 2u) ? nb4.y : -1, (m & 4u) ? nb4.z : -1,
                     (m & 8u) ? nb4.w : -1);
}

__device__ __forceinline__ int4 residual_in_arcs(const SolveView& g, uint32_t u, uint32_t* arcs)
{
    // written by this relabel's seed sweep, or derived from u's own rows
    const int4 r = (g.inrow || g.inm) ? in_arcs_written(g, u) : in_arc_row(g, u);
    *arcs = (uint32_t)(r.x >= 0) | ((uint32_t)(r.y >= 0) << 1) | ((uint32_t)(r.z >= 0) << 2) |
            ((uint32_t)(r.w >= 0) << 3);
    return r;
}

// One top-down BFS level L over cnt frontier nodes: each frontier node u
// (height L) labels every unvisited neighbor v with a residual arc v->u as
// L+1 (.cu:103-139) and appends it to the next frontier, and to the active
// queue when it holds excess.  `first` is the thread's first entry (prefetch_entry).
__device__ __forceinline__ void bfs_level_body(const SolveView& g, uint32_t L, uint32_t cnt,
                                               uint32_t first, uint32_t* s_fr, uint32_t* s_act,
                                               uint32_t* s_m, unsigned long long& visits)
{
    Ctl* ctl = g.ctl;
    const uint32_t* in = (L & 1) ? g.fr[1] : g.fr[0];
    uint32_t* out = (L & 1) ? g.fr[0] : g.fr[1];
    uint32_t* gcnt = &ctl->bfs_cnt[(L + 1) % 3];
    const uint32_t newh = L + 1u;
    const bool eager = cnt <= BFS_EAGER_MAX;
    for (uint32_t it = 0; it * (gridDim.x * DTPB) < cnt; ++it) {
        const uint32_t i = queue_index(it, cnt);
        if (i < cnt) {
            const uint32_t u = (it == 0 && cnt <= SPREAD_MAX) ? first : __ldcg(in + i);
            uint32_t arcs;
            const int4 nb4 = residual_in_arcs(g, u, &arcs);
            const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
            bool arc[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) arc[k] = (arcs >> k) & 1u;
            ++visits;
            if (eager) {
                // small frontier (latency bound): the heights and excesses of
                // the neighbours with an arc into u are loaded at once, one
                // round trip, then tested
                uint32_t hv[4];
                long long xv[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    hv[k] = arc[k] ? ldcg(g.height + nb[k]) : 0u;
                    xv[k] = arc[k] ? ldcg(g.excess + nb[k]) : 0ll;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int v = nb[k];
                    if (!arc[k] || hv[k] != UNVIS) continue;
                    if (atomicCAS(g.height + v, UNVIS, newh) == UNVIS) {
                        s_fr[atomicAdd(&s_m[0], 1u)] = (uint32_t)v;
                        if (newh < g.n && xv[k] > 0) s_act[atomicAdd(&s_m[1], 1u)] = (uint32_t)v;
                    }
                }
            } else {
                // large frontier (traffic bound): most neighbors are already
                // labeled, so an excess is read only for a node labelled here
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int v = nb[k];
                    if (!arc[k]) continue;
                    if (ldcg(g.height + v) != UNVIS) continue;
                    if (atomicCAS(g.height + v, UNVIS, newh) == UNVIS) {
                        s_fr[atomicAdd(&s_m[0], 1u)] = (uint32_t)v;
                        if (newh < g.n && ldcg(g.excess + v) > 0) s_act[atomicAdd(&s_m[1], 1u)] = (uint32_t)v;
                    }
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[2] = s_m[0]; s_m[3] = s_m[1]; s_m[0] = 0; s_m[1] = 0;
            s_m[4] = s_m[2] ? atomicAdd(gcnt, s_m[2]) : 0u;
            s_m[5] = s_m[3] ? atomicAdd(&ctl->act_cnt[0], s_m[3]) : 0u;
        }
        __syncthreads();
        flush_stage(s_fr, s_m[2], s_m[4], out, g.n, ctl);
        flush_stage(s_act, s_m[3], s_m[5], g.act[0], g.n, ctl);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(DTPB) k_bfs_seed(SolveView g)
{
    __shared__ uint32_t s_fr[DTPB * SWEEP_UNROLL], s_act[DTPB * SWEEP_UNROLL];
    __shared__ uint32_t s_m[8];
    if (threadIdx.x == 0) { s_m[0] = 0; s_m[1] = 0; }
    __syncthreads();
    bfs_seed_body<true>(g, s_fr, s_act, s_m);
}

__global__ void __launch_bounds__(DTPB) k_bfs_level(SolveView g, uint32_t L)
{
    __shared__ uint32_t s_fr[DTPB * 4], s_act[DTPB * 4];
    __shared__ uint32_t s_m[8];
    __shared__ unsigned long long s_red[DTPB / 32];
    Ctl* ctl = g.ctl;
    const uint32_t first = prefetch_entry((L & 1) ? g.fr[1] : g.fr[0], g.n);
    const uint32_t cnt = min(ldcg(&ctl->bfs_cnt[L % 3]), g.n);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->bfs_cnt[(L + 2) % 3] = 0u;
        if (cnt == 0) ctl->bfs_done = 1u;
        else atomicAdd(&ctl->bfs_levels, 1u);
    }
    if (cnt == 0) return;
    unsigned long long visits = 0;
    if (threadIdx.x == 0) { s_m[0] = 0; s_m[1] = 0; }
    __syncthreads();
    bfs_level_body(g, L, cnt, first, s_fr, s_act, s_m, visits);
    const unsigned long long vs = warp_block_sum(visits, s_red);
    if (threadIdx.x == 0 && vs) atomicAdd(&ctl->bfs_visits, vs);
}

struct Work {
    unsigned long long visits = 0, pushes = 0, relabels = 0, sink = 0;
};

// Discharge one active node for up to local_steps push/relabel steps
// (.cu:185-313).  Pushes go to residual arcs whose neighbor is lower,
// lowest first; the sink (height 0) is used when h == 1.  The relabel
// lifts v to 1 + the lowest residual neighbor.  Neighbor heights are read
// once per visit; stale values only cost work, never exactness (see the
// file comment).
// Where a discharge puts the nodes that become (or stay) active: the
// block's shared staging area while it has room, else straight into the next
// queue (chained discharges can stage more than a fixed share per thread).
struct Stage {
    uint32_t* buf;
    uint32_t* cnt;      // shared: entries claimed this block iteration
    uint32_t cap;
    uint32_t* gcnt;     // the next queue's counter
    uint32_t* out;      // the next queue
};

__device__ __forceinline__ void stage_push(const SolveView& g, const Stage& st, uint32_t u)
{
    const uint32_t idx = atomicAdd(st.cnt, 1u);
    if (idx < st.cap) {
        st.buf[idx] = u;
        return;
    }
    const uint32_t pos = atomicAdd(st.gcnt, 1u);
    if (pos < g.n) st.out[pos] = u;
    else raise_error(g.ctl, (int)GPUPR_ERR_INVARIANT);
}

// One BFS step of the persistent engine, label-correcting: a frontier node u
// with label h(u) gives every neighbor v with a residual arc v->u and a label
// above h(u)+1 (UNVIS included) the label h(u)+1 by atomicMin.  The first
// label a node gets queues it (the active queue is built after the BFS,
// active_sweep_body); with `propagate`, a later, lower label queues it again,
// so that its neighbors are relabelled from it.  With hops > 1 (short frontiers)
// the thread goes on from one node it labelled, up to `hops` nodes in a row,
// so one step, one grid barrier, covers several levels of a thin frontier; a
// node reached first by a longer path is lowered when a shorter one reaches
// it.  While every improvement propagates the labels converge to BFS
// distances (every label a node ends with was expanded), and reachability,
// which decides the end of the solve and the partition, is exact in any
// case: every labelled node is expanded at least once.  A step processes at
// most hops * cnt nodes and each queues at most 4, so the caller enables
// `propagate` only while 4 * hops * cnt <= n (the queues hold n); without it
// only first labels queue a node, at most once.  Until a chained step has run
// in this BFS every frontier node is labelled L (`exact`), and u's label is
// not read.
__device__ __forceinline__ void bfs_step_body(const SolveView& g, uint32_t L, uint32_t cnt,
                                              uint32_t first, uint32_t* s_fr,
                                              uint32_t stage_cap, uint32_t* s_m,
                                              unsigned long long& visits, int hops, bool propagate,
                                              bool exact)
{
    Ctl* ctl = g.ctl;
    const uint32_t* in = (L & 1) ? g.fr[1] : g.fr[0];
    uint32_t* out = (L & 1) ? g.fr[0] : g.fr[1];
    uint32_t* gcnt = &ctl->bfs_cnt[(L + 1) % 3];
    const Stage sf{s_fr, &s_m[0], stage_cap, gcnt, out};
    for (uint32_t it = 0; it * (gridDim.x * DTPB) < cnt; ++it) {
        const uint32_t i = queue_index(it, cnt);
        if (i < cnt) {
            uint32_t u = (it == 0 && cnt <= SPREAD_MAX) ? first : __ldcg(in + i);
            uint32_t hu = exact ? L : ldcg(g.height + u);
            uint32_t arcs;
            int4 nb4 = residual_in_arcs(g, u, &arcs);
            for (int hop = 1; hu < g.n; ++hop) {   // a queued node is labelled (< n)
                const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
                const uint32_t cand = hu + 1u;
                uint32_t next = UNVIS;
                ++visits;
                // the labels of the neighbours with an arc into u, loaded at
                // once (one round trip), then lowered where above cand
                uint32_t hv[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) hv[k] = ((arcs >> k) & 1u) ? ldcg(g.height + nb[k]) : 0u;
                // the chain's next node is normally the first neighbour that
                // passes the label test: its in-arc row is loaded together
                // with the label atomics, not after them
                int pre_v = -1;
#pragma unroll
                for (int k = 3; k >= 0; --k)
                    if (((arcs >> k) & 1u) && hv[k] > cand) pre_v = nb[k];
                int4 pre = make_int4(-1, -1, -1, -1);
                if ((g.inrow || g.inm) && hop < hops && pre_v >= 0) pre = in_arcs_written(g, pre_v);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int v = nb[k];
                    if (!((arcs >> k) & 1u) || hv[k] <= cand) continue;
                    const uint32_t old = atomicMin(g.height + v, cand);
                    if (g.bottom_up && old == UNVIS) atomicAdd(&s_m[6], 1u);   // a first label
                    if (old <= cand || (old != UNVIS && !propagate)) continue;
                    if (hop < hops && next == UNVIS) next = (uint32_t)v;
                    else stage_push(g, sf, (uint32_t)v);
                }
                if (next == UNVIS) break;
                u = next;
                hu = cand;
                if ((g.inrow || g.inm) && (int)next == pre_v) {
                    nb4 = pre;
                    arcs = (uint32_t)(pre.x >= 0) | ((uint32_t)(pre.y >= 0) << 1) |
                           ((uint32_t)(pre.z >= 0) << 2) | ((uint32_t)(pre.w >= 0) << 3);
                } else {
                    nb4 = residual_in_arcs(g, u, &arcs);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[2] = min(s_m[0], stage_cap);
            s_m[0] = 0;
            s_m[4] = s_m[2] ? atomicAdd(gcnt, s_m[2]) : 0u;
            if (g.bottom_up && s_m[6]) {
                atomicAdd(&ctl->lab_cnt[(L + 1) % 3], s_m[6]);
                s_m[6] = 0;
            }
        }
        __syncthreads();
        flush_stage(s_fr, s_m[2], s_m[4], out, g.n, ctl);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Tiled relabels (persistent engine).  A frontier step costs a grid barrier
// and a few dependent round trips per node however few nodes it labels, and a
// relabel of the benchmark graph takes ~300 of them.  Here the nodes are cut
// into tiles of RELABEL_TILE consecutive ids (node order is spatial, so most
// arcs stay inside a tile); a tile step gives every queued tile to one block,
// which loads the tile's labels and in-tile arcs into shared memory, lowers
// the labels from the tile's arcs into other tiles, runs the BFS inside the
// tile from the nodes that went down, in rounds of shared-memory worklists
// with block syncs, writes the labels that went down and
// queues, for the next step, every other tile with a node whose arc into a
// lowered node now offers a label below its own.  Labels only go down and
// each is the length of a real path to the sink; when a step's queue is empty
// no residual arc u -> v has h(u) > h(v) + 1, so the labels are the exact
// BFS distances and reachability is exact.  Each tile is written by one block
// in a step (the stamps keep a tile once per queue); labels read from other
// tiles may be older than the last write, which only re-queues a tile.
// ---------------------------------------------------------------------------
static_assert(RELABEL_TILE == DTPB * 8u, "a tile's labels fill the solver's staging buffer");

// Shared memory of one tile, after the solver's static staging buffer (which
// holds the tile's labels): per node the tile offsets of its in-arc sources
// inside the tile (four 16-bit offsets, 0xFFFF = none), its arc mask, a flag
// "label went down", and a list of 16-bit entries: the (node, slot) pairs
// whose arc leaves the tile (node << 2 | slot), or, while the BFS inside the
// tile runs, two worklists of nodes.  A tile's neighbour rows are read once,
// coalesced, per processing.
constexpr uint32_t TILE_LIST_CAP = 2u * RELABEL_TILE;
constexpr size_t TILE_SMEM = (size_t)RELABEL_TILE * 8u       // in-tile in-arc sources
                             + (size_t)RELABEL_TILE           // arc masks
                             + (size_t)RELABEL_TILE           // lowered flags
                             + (size_t)TILE_LIST_CAP * 2u;    // list / worklists
struct TileSmem {
    uint2* tin;
    uint8_t* am;
    uint8_t* low;
    uint16_t* list;
};
// Nodes one thread may take in a row in a round of the BFS inside a tile.
constexpr int TILE_CHAIN = 4;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Index for this lane's entry in a shared list whose size is *s_cnt, one
// shared atomic per warp; every active lane calls it, `want` or not.
__device__ __forceinline__ uint32_t warp_list_index(bool want, uint32_t* s_cnt)
{
    const unsigned act = __activemask();
    const unsigned bal = __ballot_sync(act, want);
    if (!bal) return 0xFFFFFFFFu;
    const int leader = __ffs(bal) - 1;
    const int lane = (int)(threadIdx.x & 31u);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(s_cnt, (uint32_t)__popc(bal));
    base = __shfl_sync(act, base, leader);
    return want ? base + (uint32_t)__popc(bal & ((1u << lane) - 1u)) : 0xFFFFFFFFu;
}

// One tile of tile step `step`, by the whole block.  s_lab: RELABEL_TILE
// labels; s_tc: four shared words (list and worklist sizes, overflow
// flags).  In the first step of a relabel (`first`) every labelled node of
// the tile announces its label to the other tiles: a seed is labelled by the
// seed sweep, before the step, so its label never goes down here.
__device__ __forceinline__ void tile_relabel(const SolveView& g, uint32_t t, uint32_t step, bool first,
                                             uint32_t* s_lab, const TileSmem& sm, uint32_t* s_tc,
                                             unsigned long long& writes, unsigned long long& levels)
{
    const uint32_t b = t << RELABEL_TILE_SHIFT;
    const uint32_t m = min(RELABEL_TILE, g.n - b);
    const int4* rows = g.nbr + b;
    // ---- the tile's labels and masks, 16 bytes a copy, all in flight ----
    const uint32_t m4 = m >> 2, m16 = m >> 4;   // whole 16-byte chunks inside the arrays
    for (uint32_t c = threadIdx.x; c < m4; c += DTPB) cp_async16(s_lab + 4u * c, g.height + b + 4u * c);
    for (uint32_t c = threadIdx.x; c < m16; c += DTPB) cp_async16(sm.am + 16u * c, g.arcm + b + 16u * c);
    for (uint32_t j = 4u * m4 + threadIdx.x; j < m; j += DTPB) s_lab[j] = ldcg(g.height + b + j);
    for (uint32_t j = 16u * m16 + threadIdx.x; j < m; j += DTPB) sm.am[j] = __ldcg(g.arcm + b + j);
    for (uint32_t j = threadIdx.x; j < m; j += DTPB) sm.low[j] = 0u;
    if (threadIdx.x < 4) s_tc[threadIdx.x] = 0u;
    cp_async_wait_all();
    __syncthreads();
    // ---- one pass over the rows (four rows of a thread in flight at once):
    // in-tile in-arc sources, and the arcs into other tiles listed ----
    for (uint32_t j0 = threadIdx.x; j0 < m; j0 += 4u * DTPB) {
        int4 rr[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t j = j0 + (uint32_t)k * DTPB;
            rr[k] = (j < m && sm.am[j]) ? __ldg(rows + j) : make_int4(-1, -1, -1, -1);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t j = j0 + (uint32_t)k * DTPB;
            if (j >= m) break;   // j grows with k: the lanes past m stay past it
            const uint32_t am = sm.am[j];
            const int nb[4] = {rr[k].x, rr[k].y, rr[k].z, rr[k].w};
            uint32_t loc[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t off = (uint32_t)nb[q] - b;
                loc[q] = (((am >> (4 + q)) & 1u) && off < m) ? off : 0xFFFFu;
                const bool x = ((am >> q) & 1u) && off >= m;
                const uint32_t i = warp_list_index(x, &s_tc[0]);
                if (x && i < TILE_LIST_CAP) sm.list[i] = (uint16_t)((j << 2) | (uint32_t)q);
                else if (x) {   // list full: this one at once
                    const uint32_t hv = ldcg(g.height + nb[q]);
                    if (hv != UNVIS && atomicMin(s_lab + j, hv + 1u) > hv + 1u) sm.low[j] = 1u;
                }
            }
            sm.tin[j] = make_uint2(loc[0] | (loc[1] << 16), loc[2] | (loc[3] << 16));
        }
    }
    __syncthreads();
    // ---- lower each listed source node from the other tile's label, all
    // loads of a thread in flight at once ----
    const uint32_t npull = min(s_tc[0], TILE_LIST_CAP);
    for (uint32_t i0 = 0; i0 < npull; i0 += 4u * DTPB) {
        uint32_t e[4], hv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t i = i0 + (uint32_t)k * DTPB + threadIdx.x;
            e[k] = i < npull ? sm.list[i] : 0xFFFFFFFFu;
            hv[k] = UNVIS;
            if (e[k] != 0xFFFFFFFFu) {
                const int4 r = __ldg(rows + (e[k] >> 2));
                const int nb[4] = {r.x, r.y, r.z, r.w};
                hv[k] = ldcg(g.height + nb[e[k] & 3u]);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (hv[k] == UNVIS) continue;
            const uint32_t j = e[k] >> 2;
            if (atomicMin(s_lab + j, hv[k] + 1u) > hv[k] + 1u) sm.low[j] = 1u;
        }
    }
    // ---- the BFS inside the tile, by worklists: a node whose label went down
    // (or, in the first step, every labelled node) offers label + 1 to its
    // in-tile in-arc sources; a source that takes it is expanded next by the
    // same thread (up to TILE_CHAIN in a row) or listed for the next round.
    // Only the tile's own block writes its labels, so the tile was at a
    // fixpoint after its last processing and only these nodes can move it.
    // A list that overflows makes the next round expand every node. ----
    __syncthreads();   // the pull list is consumed: its space holds the worklists
    if (threadIdx.x == 0) s_tc[0] = 0u;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < m; j += DTPB) {
        const bool x = sm.low[j] || (first && s_lab[j] != UNVIS);
        const uint32_t i = warp_list_index(x, &s_tc[0]);
        if (x) sm.list[i] = (uint16_t)j;   // at most m entries
    }
    __syncthreads();
    for (uint32_t r = 0;; ++r) {
        const uint32_t c = min(s_tc[r & 1u], RELABEL_TILE);
        const bool full = s_tc[2u + (r & 1u)] != 0u;
        __syncthreads();   // every thread has read this round's counts
        if (c == 0u && !full) break;
        if (r > g.n + 2u) {   // every round lowers a label: a broken invariant
            if (threadIdx.x == 0) raise_error(g.ctl, (int)GPUPR_ERR_INVARIANT);
            break;
        }
        const uint32_t nx = (r + 1u) & 1u;
        if (threadIdx.x == 0) {
            s_tc[nx] = 0u;
            s_tc[2u + nx] = 0u;
        }
        __syncthreads();
        const uint32_t cnt = full ? m : c;
        for (uint32_t i = threadIdx.x; i < cnt; i += DTPB) {
            uint32_t v = full ? i : sm.list[(r & 1u) * RELABEL_TILE + i];
            for (int hop = 1;; ++hop) {
                const uint32_t nl = s_lab[v] + 1u;
                if (nl == 0u) break;   // unlabelled (UNVIS + 1 wraps)
                const uint2 p = sm.tin[v];
                const uint32_t src[4] = {p.x & 0xFFFFu, p.x >> 16, p.y & 0xFFFFu, p.y >> 16};
                uint32_t old[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)   // four independent atomics in flight
                    old[q] = src[q] != 0xFFFFu ? atomicMin(s_lab + src[q], nl) : 0u;
                uint32_t next = 0xFFFFFFFFu;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t u = src[q];
                    if (old[q] <= nl) continue;
                    sm.low[u] = 1u;
                    if (next == 0xFFFFFFFFu && hop < TILE_CHAIN) {
                        next = u;
                        continue;
                    }
                    const uint32_t k = atomicAdd(&s_tc[nx], 1u);
                    if (k < RELABEL_TILE) sm.list[nx * RELABEL_TILE + k] = (uint16_t)u;
                    else s_tc[2u + nx] = 1u;
                }
                if (next == 0xFFFFFFFFu) break;
                v = next;
            }
        }
        ++levels;
        __syncthreads();
    }
    // ---- write the labels that went down; list their arcs from other tiles ----
    if (threadIdx.x == 0) s_tc[0] = 0u;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < m; j += DTPB) {
        const uint32_t h = s_lab[j];
        const bool lowered = sm.low[j] != 0u;
        if (lowered) {
            g.height[b + j] = h;
            ++writes;
        }
        // in-arcs from other tiles: an in-arc bit whose source is not in the tile
        const uint2 p = sm.tin[j];
        const uint32_t src[4] = {p.x & 0xFFFFu, p.x >> 16, p.y & 0xFFFFu, p.y >> 16};
        const uint32_t in = (lowered || (first && h != UNVIS)) ? (uint32_t)(sm.am[j] >> 4) : 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const bool x = ((in >> q) & 1u) && src[q] == 0xFFFFu;
            const uint32_t i = warp_list_index(x, &s_tc[0]);
            if (x && i < TILE_LIST_CAP) sm.list[i] = (uint16_t)((j << 2) | (uint32_t)q);
            else if (x) {   // list full: this one at once
                const int4 r = __ldg(rows + j);
                const int nb[4] = {r.x, r.y, r.z, r.w};
                if (ldcg(g.height + nb[q]) > h + 1u)
                    queue_tile(g, (uint32_t)nb[q] >> RELABEL_TILE_SHIFT, step + 1u);
            }
        }
    }
    __syncthreads();
    // ---- queue the other tiles whose node now has a shorter way out ----
    const uint32_t nnote = min(s_tc[0], TILE_LIST_CAP);
    for (uint32_t i0 = 0; i0 < nnote; i0 += 4u * DTPB) {
        uint32_t w[4], hw[4], e[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t i = i0 + (uint32_t)k * DTPB + threadIdx.x;
            e[k] = i < nnote ? sm.list[i] : 0xFFFFFFFFu;
            w[k] = 0xFFFFFFFFu;
            hw[k] = 0u;
            if (e[k] != 0xFFFFFFFFu) {
                const int4 r = __ldg(rows + (e[k] >> 2));
                const int nb[4] = {r.x, r.y, r.z, r.w};
                w[k] = (uint32_t)nb[e[k] & 3u];
                hw[k] = ldcg(g.height + w[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (w[k] == 0xFFFFFFFFu || hw[k] <= s_lab[e[k] >> 2] + 1u) continue;
            const uint32_t tw = w[k] >> RELABEL_TILE_SHIFT;
            if (ldcg(g.tile_stamp + tw) < step + 1u) queue_tile(g, tw, step + 1u);
        }
    }
    __syncthreads();   // the shared tile is the next tile's
}

// One frontier node u with label hu, expanded: every neighbour v with a
// residual arc v -> u and a label above hu + 1 (UNVIS included) is lowered
// to hu + 1 by atomicMin and staged when that is its first label or, with
// `propagate`, a lower one (the rule of bfs_step_body without the chain).
// With direction-optimizing relabels, first labels are counted in s_m[6].
__device__ __forceinline__ void bfs_expand_one(const SolveView& g, uint32_t u, uint32_t hu,
                                               const Stage& st, bool propagate,
                                               unsigned long long& visits, uint32_t* s_m)
{
    uint32_t arcs;
    const int4 nb4 = residual_in_arcs(g, u, &arcs);
    const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
    const uint32_t cand = hu + 1u;
    ++visits;
    uint32_t hv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) hv[k] = ((arcs >> k) & 1u) ? ldcg(g.height + nb[k]) : 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!((arcs >> k) & 1u) || hv[k] <= cand) continue;
        const uint32_t old = atomicMin(g.height + nb[k], cand);
        if (g.bottom_up && old == UNVIS) atomicAdd(&s_m[6], 1u);   // a first label
        if (old <= cand || (old != UNVIS && !propagate)) continue;
        stage_push(g, st, (uint32_t)nb[k]);
    }
}

// A BFS step of the persistent engine with block sub-levels (option
// bfs_block_levels = K > 1): each block expands its share of the frontier
// (level L), then, without a grid barrier, the nodes it labelled itself, for
// up to K - 1 more levels, breadth first, from its shared-memory stage (two
// halves of stage_cap / 2 entries, ping-pong); only the last sub-level's
// nodes, and any that overflow a half, go to the next step's queue.  Labels
// are corrected like the chained steps' (atomicMin, re-queued while
// `propagate`): a node labelled here before another block reaches it by a
// shorter path is lowered and expanded again.  Frontier entries may carry
// different labels: each expansion reads its node's label.
__device__ __forceinline__ void bfs_step_levels_body(const SolveView& g, uint32_t L, uint32_t cnt,
                                                     uint32_t first, uint32_t* s_fr,
                                                     uint32_t stage_cap, uint32_t* s_m,
                                                     unsigned long long& visits, int levels,
                                                     bool propagate, bool exact)
{
    Ctl* ctl = g.ctl;
    const uint32_t* in = (L & 1) ? g.fr[1] : g.fr[0];
    uint32_t* out = (L & 1) ? g.fr[0] : g.fr[1];
    uint32_t* gcnt = &ctl->bfs_cnt[(L + 1) % 3];
    const uint32_t half = stage_cap / 2u;
    for (uint32_t it = 0; it * (gridDim.x * DTPB) < cnt; ++it) {
        uint32_t* cur = s_fr;
        uint32_t* nxt = s_fr + half;
        {
            const Stage st{cur, &s_m[0], half, gcnt, out};
            const uint32_t i = queue_index(it, cnt);
            if (i < cnt) {
                const uint32_t u = (it == 0 && cnt <= SPREAD_MAX) ? first : __ldcg(in + i);
                bfs_expand_one(g, u, exact ? L : ldcg(g.height + u), st, propagate, visits, s_m);
            }
        }
        __syncthreads();
        for (int k = 1; k < levels; ++k) {
            const uint32_t c = min(s_m[0], half);
            __syncthreads();   // every thread has read the count
            if (c == 0u) break;
            if (threadIdx.x == 0) s_m[0] = 0u;
            __syncthreads();
            const Stage st{nxt, &s_m[0], half, gcnt, out};
            for (uint32_t j = threadIdx.x; j < c; j += DTPB) {
                const uint32_t u = cur[j];
                bfs_expand_one(g, u, ldcg(g.height + u), st, propagate, visits, s_m);
            }
            __syncthreads();
            uint32_t* tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
        if (threadIdx.x == 0) {
            s_m[2] = min(s_m[0], half);
            s_m[0] = 0;
            s_m[4] = s_m[2] ? atomicAdd(gcnt, s_m[2]) : 0u;
            if (g.bottom_up && s_m[6]) {
                atomicAdd(&ctl->lab_cnt[(L + 1) % 3], s_m[6]);
                s_m[6] = 0;
            }
        }
        __syncthreads();
        flush_stage(cur, s_m[2], s_m[4], out, g.n, ctl);
        __syncthreads();
    }
}

// Frontier entries block 0 keeps in shared memory in a tail step, and the
// most levels one tail step covers (a bound on the other blocks' barrier wait).
constexpr uint32_t TAIL_CAP = DTPB * 4u;
constexpr int TAIL_LEVELS = 4096;
// Default frontier size up to which tail steps run (0: none).
constexpr uint32_t BFS_TAIL_DEFAULT = 0u;
// Levels a block expands per BFS step from its own stage by default
// (bfs_step_levels_body).
constexpr int BFS_BLOCK_LEVELS = 16;
// Whether the persistent engine's frontier steps read in-arc masks (one byte
// per node, next to the node's neighbour row) instead of 16-byte in-arc rows
// by default.  The seed sweep then streams 41 instead of 72 bytes a node (no
// neighbour row read, one byte written instead of 16), and a BFS expansion
// reads the neighbour row and the mask byte instead of the in-arc row: the
// mask array (1 byte a node) stays largely in L2.  Measured on B200 (median of
// 7 alternating solves, cuts identical): benchmark graph 68.4 -> 67.3 ms
// (relabels 36.3 -> 35.0 ms), 3M-tet torus 1.83 -> 1.81 ms, 8M-tet open box
// 12.8 -> 12.6 ms; 15 bytes less workspace per node.
constexpr bool BFS_IN_ARC_MASKS_DEFAULT = true;
// Free nodes from which the persistent engine relabels by tiles by default.
constexpr uint32_t RELABEL_TILES_DEFAULT_MIN = 0xFFFFFFFFu;

// A tail step of the persistent engine's BFS, run by block 0 alone while the
// other blocks wait at the grid barrier: starting from level L0's frontier
// (cnt0 <= TAIL_CAP nodes), it expands level after level with the frontier in
// shared memory and block-level syncs instead of a grid barrier per level
// (the same label-correcting rule as bfs_step_body: a neighbour with an arc
// into u and a label above h(u)+1 is lowered by atomicMin and queued when
// first labelled, or when improved while 4 x frontier <= n).  It stops when a
// frontier is empty, no longer fits in shared memory or exceeds g.tail_max,
// or after TAIL_LEVELS levels; it then leaves that level's frontier in the
// global queue for it with its count, every other ring counter at zero, and
// the level in ctl->tail_L.  s_buf holds 2 * TAIL_CAP entries; s_m[10] is the
// claim counter.
__device__ void bfs_tail_body(const SolveView& g, uint32_t L0, uint32_t cnt0, uint32_t* s_buf,
                              uint32_t* s_m, unsigned long long& visits)
{
    Ctl* ctl = g.ctl;
    uint32_t* sA = s_buf;
    uint32_t* sB = s_buf + TAIL_CAP;
    const uint32_t* in0 = (L0 & 1) ? g.fr[1] : g.fr[0];
    for (uint32_t i = threadIdx.x; i < cnt0; i += DTPB) sA[i] = __ldcg(in0 + i);
    uint32_t L = L0, nA = cnt0;
    __syncthreads();
    for (int lv = 0;; ++lv) {
        // expand level L (frontier sA[0..nA)) into level L+1
        uint32_t* out = (L & 1) ? g.fr[0] : g.fr[1];   // level L+1's global queue
        const bool propagate = 4ull * nA <= (unsigned long long)g.n;
        if (threadIdx.x == 0) s_m[10] = 0u;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nA; i += DTPB) {
            const uint32_t u = sA[i];
            const uint32_t hu = ldcg(g.height + u);
            if (hu >= g.n) continue;
            uint32_t arcs;
            const int4 nb4 = residual_in_arcs(g, u, &arcs);
            const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
            const uint32_t cand = hu + 1u;
            ++visits;
            uint32_t hv[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) hv[k] = ((arcs >> k) & 1u) ? ldcg(g.height + nb[k]) : 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int v = nb[k];
                if (!((arcs >> k) & 1u) || hv[k] <= cand) continue;
                const uint32_t old = atomicMin(g.height + v, cand);
                if (old <= cand || (old != UNVIS && !propagate)) continue;
                // entries past the shared array go straight to the global queue,
                // behind room for the shared ones
                const uint32_t idx = atomicAdd(&s_m[10], 1u);
                if (idx < TAIL_CAP) sB[idx] = (uint32_t)v;
                else if (idx < g.n) out[idx] = (uint32_t)v;
                else raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
            }
        }
        __syncthreads();
        const uint32_t nB = min(s_m[10], g.n);
        ++L;
        if (nB == 0u || nB > TAIL_CAP || nB > g.tail_max || lv + 1 >= TAIL_LEVELS || L > g.n + 2u) {
            const uint32_t m = min(nB, TAIL_CAP);
            for (uint32_t i = threadIdx.x; i < m; i += DTPB) out[i] = sB[i];
            if (threadIdx.x == 0) {
                for (int k = 0; k < 3; ++k) ctl->bfs_cnt[k] = 0u;
                ctl->bfs_cnt[L % 3] = nB;
                ctl->tail_L = L;
                ctl->tail_steps += 1ull;
                ctl->tail_levels += (unsigned long long)(L - L0);
            }
            return;
        }
        uint32_t* t = sA;
        sA = sB;
        sB = t;
        nA = nB;
        __syncthreads();
    }
}

// One bottom-up step j of a direction-optimizing relabel (frontier label L):
// every candidate v of list j (cand[j % 2], size in bu_cnt[j % 3]; list 0 is
// the previous relabel's reached set, which holds every node this relabel can
// reach: a push runs only between reached nodes, so the reached set never
// grows) that is still unlabelled and has a residual arc to a labelled
// neighbour takes 1 + the lowest such label and joins the next frontier;
// the others stay candidates in list j+1.  v's own rows give the arcs v->u,
// so only the neighbours' labels are gathered.  s_fr and s_keep hold
// stage_cap entries each; s_m[0,2,4] stage the frontier, s_m[7..9] the list.
__device__ __forceinline__ void bfs_bottom_up_body(const SolveView& g, uint32_t L, uint32_t j,
                                                   uint32_t* s_fr, uint32_t* s_keep, uint32_t stage_cap,
                                                   uint32_t* s_m, unsigned long long& visits)
{
    Ctl* ctl = g.ctl;
    const uint32_t* in = g.cand[j & 1u];
    uint32_t* keep = g.cand[(j + 1u) & 1u];
    uint32_t* kcnt = &ctl->bu_cnt[(j + 1u) % 3u];
    uint32_t* out = (L & 1) ? g.fr[0] : g.fr[1];
    uint32_t* gcnt = &ctl->bfs_cnt[(L + 1) % 3];
    const uint32_t cnt = min(vload(&ctl->bu_cnt[j % 3u]), g.n);
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->bu_cnt[(j + 2u) % 3u] = 0u;
    for (uint32_t it = 0; it * (gridDim.x * DTPB) < cnt; ++it) {
        const uint32_t i = (it * gridDim.x + blockIdx.x) * DTPB + threadIdx.x;   // node order
        if (i < cnt) {
            const uint32_t v = __ldcg(in + i);
            if (v < g.n && ldcg(g.height + v) == UNVIS) {
                const int4 nb4 = __ldg(g.nbr + v);
                const uint4 r4 = __ldcg(reinterpret_cast<const uint4*>(g.res) + v);
                const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
                const uint32_t r[4] = {r4.x, r4.y, r4.z, r4.w};
                uint32_t hv[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) hv[k] = (nb[k] >= 0 && r[k] != 0u) ? ldcg(g.height + nb[k]) : UNVIS;
                const uint32_t best = min(min(hv[0], hv[1]), min(hv[2], hv[3]));
                ++visits;
                if (best != UNVIS) {
                    atomicMin(g.height + v, best + 1u);
                    s_fr[atomicAdd(&s_m[0], 1u)] = v;
                } else {
                    s_keep[atomicAdd(&s_m[7], 1u)] = v;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[2] = min(s_m[0], stage_cap);
            s_m[0] = 0;
            s_m[4] = s_m[2] ? atomicAdd(gcnt, s_m[2]) : 0u;
            if (s_m[2]) atomicAdd(&ctl->lab_cnt[(L + 1) % 3], s_m[2]);
            s_m[8] = min(s_m[7], stage_cap);
            s_m[7] = 0;
            s_m[9] = s_m[8] ? atomicAdd(kcnt, s_m[8]) : 0u;
        }
        __syncthreads();
        flush_stage(s_fr, s_m[2], s_m[4], out, g.n, ctl);
        flush_stage(s_keep, s_m[8], s_m[9], keep, g.n, ctl);
        __syncthreads();
    }
}

// Returns the node to discharge next in the same round (chaining: a node
// whose excess this discharge moved from 0 up is owned by this thread, and
// instead of queueing it for the next round the thread may carry on with
// it, so excess can travel several hops per round), or UNVIS.
template <bool kAgg>
__device__ __forceinline__ uint32_t discharge_node(const SolveView& g, uint32_t v, const Stage& st,
                                                   bool may_chain, Work& w)
{
    const uint32_t n = g.n;
    // every load of the node's own state is issued before any test, so they
    // share one round trip to L2 (a queued node nearly always passes both
    // tests); L2 loads because a previous owner may have run on another SM
    uint32_t h = ldcg(g.height + v);
    long long ex = ldcg(g.excess + v);
    const int4 nb4 = __ldg(g.nbr + v);
    const uint4 r4 = __ldcg(reinterpret_cast<const uint4*>(g.res) + v);
    const uint32_t rv = __ldg(g.rev + v);
    int32_t t = ldcg(g.term + v);
    if (h >= n || ex <= 0) return UNVIS;
    uint32_t next = UNVIS;
    const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
    uint32_t r[4] = {r4.x, r4.y, r4.z, r4.w};
    uint32_t hn[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) hn[k] = (nb[k] >= 0) ? ldcg(g.height + nb[k]) : UNVIS;
    const uint32_t h0 = h;
    const int32_t t0 = t;
    long long pushed = 0;
    ++w.visits;
    for (int step = 0; step < g.local_steps; ++step) {
        if (t < 0 && h == 1u) {                       // v -> sink (.cu:220-236)
            const long long cap = -(long long)t;
            const long long d = ex < cap ? ex : cap;
            t = (int32_t)((long long)t + d);
            ex -= d;
            pushed += d;
            w.sink += (unsigned long long)d;
            ++w.pushes;
        }
        while (ex > 0) {                               // admissible pushes
            int best = -1;
            uint32_t bh = h;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (nb[k] >= 0 && r[k] != 0u && hn[k] < bh) { bh = hn[k]; best = k; }
            if (best < 0) break;
            uint32_t rb = 0u;
            int u = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k == best) { rb = r[k]; u = nb[k]; }
            const uint32_t d = (uint32_t)(ex < (long long)rb ? ex : (long long)rb);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k == best) r[k] -= d;
            ex -= d;
            pushed += d;
            const uint32_t rk = (rv >> (2 * best)) & 3u;
            atomicSub(g.res + (size_t)v * 4u + best, d);
            atomicAdd(g.res + (size_t)u * 4u + rk, d);
            bool owner;
            if (kAgg) {
                // lanes pushing to the same neighbour now add their amounts in
                // one atomic, issued by the group's first lane, which takes
                // ownership when the neighbour's excess was zero
                const cg::coalesced_group active = cg::coalesced_threads();
                const cg::coalesced_group same = cg::labeled_partition(active, (unsigned)u);
                const unsigned long long sum = cg::reduce(same, (unsigned long long)d,
                                                          cg::plus<unsigned long long>());
                owner = same.thread_rank() == 0 &&
                        atomicAdd(reinterpret_cast<unsigned long long*>(g.excess + u), sum) == 0ull;
            } else {
                owner = atomicAdd(reinterpret_cast<unsigned long long*>(g.excess + u),
                                  (unsigned long long)d) == 0ull;
            }
            if (owner) {
                if (may_chain && next == UNVIS) next = (uint32_t)u;
                else stage_push(g, st, (uint32_t)u);
            }
            ++w.pushes;
        }
        if (ex <= 0) break;
        uint32_t mh = (t < 0) ? 0u : UNVIS;            // relabel (.cu:274-301)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (nb[k] >= 0 && r[k] != 0u && hn[k] < mh) mh = hn[k];
        ++w.relabels;
        if (mh == UNVIS) { h = UNVIS; break; }
        h = mh + 1u;
        if (h >= n) break;
    }
    if (h != h0) g.height[v] = h;
    if (t != t0) g.term[v] = t;
    long long now = ex;
    if (pushed) {
        const unsigned long long old = atomicAdd(reinterpret_cast<unsigned long long*>(g.excess + v),
                                                 (unsigned long long)(-pushed));
        now = (long long)old - pushed;
    }
    if (now > 0 && h < n) stage_push(g, st, v);   // keeps ownership
    return next;
}

// One discharge round over cnt active nodes: discharge each, stage the nodes
// that become (or stay) active, append them to the next active queue.
// `first` is the thread's first entry (prefetch_entry).
template <bool kAgg>
__device__ __forceinline__ void discharge_body(const SolveView& g, uint32_t round, uint32_t cnt,
                                               uint32_t first, uint32_t* s_buf, uint32_t stage_cap,
                                               uint32_t* s_m, Work& w)
{
    Ctl* ctl = g.ctl;
    const uint32_t* in = (round & 1) ? g.act[1] : g.act[0];
    uint32_t* out = (round & 1) ? g.act[0] : g.act[1];
    uint32_t* gcnt = &ctl->act_cnt[(round + 1) % 3];
    const Stage st{s_buf, &s_m[0], stage_cap, gcnt, out};
    const int hops = cnt <= g.chain_max_active ? g.chain_hops : 1;
    for (uint32_t it = 0; it * (gridDim.x * DTPB) < cnt; ++it) {
        const uint32_t i = queue_index(it, cnt);
        if (i < cnt) {
            uint32_t v = (it == 0 && cnt <= SPREAD_MAX) ? first : __ldcg(in + i);
            if (v < g.n) {
                for (int hop = 1;; ++hop) {
                    v = discharge_node<kAgg>(g, v, st, hop < hops, w);
                    if (v == UNVIS) break;
                }
            } else {
                raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_m[2] = min(s_m[0], stage_cap);
            s_m[0] = 0;
            s_m[4] = s_m[2] ? atomicAdd(gcnt, s_m[2]) : 0u;
        }
        __syncthreads();
        flush_stage(s_buf, s_m[2], s_m[4], out, g.n, ctl);
        __syncthreads();
    }
}

__device__ __forceinline__ void reduce_work(Ctl* ctl, const Work& w, unsigned long long bfs_visits,
                                            unsigned long long* s_red)
{
    unsigned long long x;
    x = warp_block_sum(w.visits, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(&ctl->node_visits, x);
    x = warp_block_sum(w.pushes, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(&ctl->pushes, x);
    x = warp_block_sum(w.relabels, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(&ctl->relabels, x);
    x = warp_block_sum(w.sink, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(&ctl->sink_flow, x);
    x = warp_block_sum(bfs_visits, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(&ctl->bfs_visits, x);
}

__global__ void __launch_bounds__(DTPB) k_discharge(SolveView g, uint32_t round)
{
    __shared__ uint32_t s_buf[DTPB * 5];
    __shared__ uint32_t s_m[8];
    __shared__ unsigned long long s_red[DTPB / 32];
    Ctl* ctl = g.ctl;
    const uint32_t first = prefetch_entry((round & 1) ? g.act[1] : g.act[0], g.n);
    const uint32_t cnt = min(ldcg(&ctl->act_cnt[round % 3]), g.n);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->act_cnt[(round + 2) % 3] = 0u;
        if (cnt) atomicAdd(&ctl->rounds_done, 1u);
    }
    if (cnt == 0) return;
    Work w;
    if (threadIdx.x == 0) s_m[0] = 0;
    __syncthreads();
    discharge_body<false>(g, round, cnt, first, s_buf, DTPB * 5, s_m, w);
    reduce_work(ctl, w, 0ull, s_red);
}

// ---------------------------------------------------------------------------
// Persistent engine: the whole solve in one cooperative launch.  The same
// level and round steps as above run back to back, separated by a software
// grid barrier instead of a kernel boundary, and the control decisions
// (frontier/queue empty, relabel period, work budget, round limit) are taken
// by every block from the same counters read after a barrier, so all blocks
// follow the same path.  Every barrier wait is bounded; an error or the time
// limit makes every block leave at its next barrier.
// ---------------------------------------------------------------------------
// Segmented solve: a graph in which the active sweep after an exact relabel
// found no active node is finished (its preflow is maximum and nothing in it
// changes any more), so it retires: the seeds and sweeps that follow skip its
// nodes, no BFS enters it (the graphs share no arc), and its labels from this
// relabel give its partition.  Clears the marks of the graphs that go on.
__device__ __forceinline__ void retire_graphs(const SolveView& g)
{
    for (uint32_t k = blockIdx.x * DTPB + threadIdx.x; k < g.nseg; k += gridDim.x * DTPB) {
        if (!ldcg(g.seg_live + k)) continue;
        if (ldcg(g.seg_act + k)) {
            g.seg_act[k] = 0u;
            continue;
        }
        g.seg_live[k] = 0u;
        atomicAdd(&g.ctl->segs_retired, 1u);
        atomicAdd(&g.ctl->retired_nodes,
                  (unsigned long long)(__ldg(g.seg_off + k + 1u) - __ldg(g.seg_off + k)));
    }
}

struct PersistParams {
    unsigned long long max_rounds;
    unsigned long long budget;      // node visits per discharge phase, 0 = none
    unsigned long long limit_ns;    // solve time limit
    unsigned long long wait_ns;     // bound of one barrier wait
    uint32_t relabel_rounds;        // rounds per discharge phase, 0 = none
};

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add(unsigned long long* p, unsigned long long v)
{
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid-wide barrier of the persistent engine (all blocks co-resident by the
// cooperative launch).  ctl->bar counts arrivals since the launch; a block's
// thread 0 adds its arrival with release semantics and polls with acquire
// loads until the count reaches this barrier's target (kept per block in
// `target`): one round trip to L2 to arrive, one to see the last arrival.
// An error anywhere sets BAR_ABORT, which ends every wait at once; a wait
// also ends, with GPUPR_ERR_TIMEOUT, after wait_ns, and block 0 raises the
// solve's own time limit here.
__device__ bool grid_barrier(Ctl* ctl, unsigned long long& target, unsigned long long deadline,
                             unsigned long long wait_ns, int* s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        if (blockIdx.x == 0 && gtimer() > deadline) raise_error(ctl, (int)GPUPR_ERR_TIMEOUT);
        red_release_add(&ctl->bar, 1ull);
        int ok = 1;
        unsigned long long t0 = 0;
        for (uint32_t it = 0;; ++it) {
            const unsigned long long v = ld_acquire(&ctl->bar);
            if (v & BAR_ABORT) { ok = 0; break; }
            if ((v & BAR_COUNT) >= target) break;
            // a long wait (block 0's BFS tail) polls less often, off the L2
            // slice that holds the counter
            if (it >= 2048u) __nanosleep(256);
            if ((it & 63u) == 0u) {
                const unsigned long long t = gtimer();
                if (it == 0u) t0 = t;
                else if (t - t0 > wait_ns) {
                    raise_error(ctl, (int)GPUPR_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// kAgg: warp-aggregated excess atomics in the discharge (an option).
// kTiles: tiled relabels (g.arcm set), a separate instantiation so that the
// frontier-step kernel keeps its registers.
template <bool kAgg, bool kTiles>
__global__ void __launch_bounds__(DTPB, 4) k_solve_persistent(SolveView g, PersistParams p)
{
    __shared__ __align__(16) uint32_t s_buf[DTPB * 8];   // 16-byte copies land here (tiles)
    __shared__ uint32_t s_m[12];
    __shared__ unsigned long long s_red[DTPB / 32];
    __shared__ int s_ok;
    Ctl* ctl = g.ctl;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const unsigned long long deadline = gtimer() + p.limit_ns;
    unsigned long long bar_target = 0;
    Work w;
    unsigned long long bfs_visits = 0;
    // tiled relabels: the last tile step (the same in every block), tiles and
    // nodes this block processed, labels this thread lowered
    uint32_t tstep = 0;
    unsigned long long tprocs = 0, tloads = 0, twrites = 0, tsteps = 0, tlevels = 0;
    // tiled relabels: the tile's rows, masks, flags and list (TILE_SMEM bytes
    // of dynamic shared memory; none in the other instantiations)
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ uint32_t s_tc[kTiles ? 4 : 1];
    TileSmem tsm{};
    if (kTiles) {
        tsm.tin = reinterpret_cast<uint2*>(s_dyn);
        tsm.am = s_dyn + (size_t)RELABEL_TILE * 8u;
        tsm.low = tsm.am + RELABEL_TILE;
        tsm.list = reinterpret_cast<uint16_t*>(tsm.low + RELABEL_TILE);
    }
    if (threadIdx.x < 12) s_m[threadIdx.x] = 0u;
    // phase clock of block 0, read after each phase's closing barrier:
    // s_clk = {BFS, active sweep, discharge, last mark} (shared memory, so it
    // holds no registers through the solve)
    __shared__ unsigned long long s_clk[4];
    __shared__ unsigned long long s_step_ns[3];
    __shared__ uint32_t s_step_cnt[3];
    __shared__ unsigned long long s_dr_ns[3], s_dr_t0;
    __shared__ uint32_t s_dr_cnt[3];
    auto lap = [&](int phase) {
        if (lead) {
            const unsigned long long t = gtimer();
            s_clk[phase] += t - s_clk[3];
            s_clk[3] = t;
        }
    };
    constexpr uint32_t CH = DTPB * SWEEP_UNROLL;
    for (uint32_t base = blockIdx.x * CH; base < g.n; base += gridDim.x * CH) {
        int32_t t[SWEEP_UNROLL];
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            t[j] = v < g.n ? ldcg(g.term + v) : 0;
        }
#pragma unroll
        for (int j = 0; j < SWEEP_UNROLL; ++j) {
            const uint32_t v = base + j * DTPB + threadIdx.x;
            if (v < g.n) g.excess[v] = t[j] > 0 ? (long long)t[j] : 0ll;   // source arc saturated (.cu:69-83)
        }
    }
    if (grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok)) {
        unsigned long long rounds_total = 0;
        uint32_t levels_total = 0, relabels = 0;
        bool ok = true;
        if (lead) {
            s_clk[0] = s_clk[1] = s_clk[2] = 0ull;
            s_clk[3] = gtimer();
            for (int k = 0; k < 3; ++k) { s_step_ns[k] = 0ull; s_step_cnt[k] = 0u; s_dr_ns[k] = 0ull; s_dr_cnt[k] = 0u; }
        }
        while (ok) {
            // ---- global relabel (label-correcting steps, reachability exact) ----
            bfs_seed_body<false>(g, s_buf, s_buf + DTPB * 4, s_m, kTiles ? tstep + 1u : 0u);
            if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
            const uint32_t S0 = tstep + 1u;   // the seeds' tile step
            while (kTiles) {
                // ---- tile steps (tiled relabels) ----
                const uint32_t S = ++tstep;
                const uint32_t cnt = min(vload(&ctl->bfs_cnt[S % 3u]), g.ntiles);
                if (cnt == 0) break;
                if (lead) ctl->bfs_cnt[(S + 2u) % 3u] = 0u;
                const uint32_t* tq = (S & 1u) ? g.fr[1] : g.fr[0];
                for (uint32_t i = blockIdx.x; i < cnt; i += gridDim.x) {
                    const uint32_t t = __ldcg(tq + i);
                    if (t >= g.ntiles) {   // queue entries are tile ids by construction
                        if (threadIdx.x == 0) raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
                        continue;
                    }
                    tile_relabel(g, t, S, S == S0, s_buf, tsm, s_tc, twrites, tlevels);
                    ++tprocs;
                    tloads += min(RELABEL_TILE, g.n - (t << RELABEL_TILE_SHIFT));
                }
                if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
                ++levels_total;
                ++tsteps;
            }
            if (!ok) break;
            uint32_t L = 1;
            bool exact = true;   // no chained step yet: every frontier node is labelled L
            uint32_t labelled = 0, bu_j = 0;
            for (; !kTiles;) {
                const uint32_t first = prefetch_entry((L & 1) ? g.fr[1] : g.fr[0], g.n);
                const uint32_t cnt = min(vload(&ctl->bfs_cnt[L % 3]), g.n);
                if (cnt == 0) break;
                if (lead) ctl->bfs_cnt[(L + 2) % 3] = 0u;
                const unsigned long long t_step = lead ? gtimer() : 0ull;
                // every decision below is the same in every block: it depends
                // on counters completed before the last barrier
                bool bottom_up = false;
                if (g.bottom_up) {
                    labelled += vload(&ctl->lab_cnt[L % 3]);
                    if (lead) ctl->lab_cnt[(L + 2) % 3] = 0u;
                    const uint32_t cc = vload(&ctl->cand_cnt);
                    const uint32_t rem = cc > labelled ? cc - labelled : 0u;
                    bottom_up = cc != 0u && (float)rem <= g.bu_ratio * (float)cnt;
                }
                if (!g.bottom_up && g.tail_max && cnt <= g.tail_max) {
                    // a short frontier: block 0 runs the next levels alone
                    if (blockIdx.x == 0) bfs_tail_body(g, L, cnt, s_buf, s_m, bfs_visits);
                    exact = false;
                    if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
                    if (lead) {
                        s_step_ns[0] += gtimer() - t_step;
                        ++s_step_cnt[0];
                    }
                    const uint32_t Lt = vload(&ctl->tail_L);
                    levels_total += Lt - L;
                    L = Lt;
                    if (L > g.n + 2u) {
                        if (lead) raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
                        ok = false;
                        break;
                    }
                    continue;
                }
                if (bottom_up) {
                    bfs_bottom_up_body(g, L, bu_j, s_buf, s_buf + DTPB * 4, DTPB * 4, s_m, bfs_visits);
                    ++bu_j;
                    exact = false;
                    if (lead) ++ctl->bu_steps;
                } else if (g.bfs_block_levels > 1) {
                    // expansions this step: the frontier, then per block and
                    // pass at most one stage half per sub-level
                    const unsigned long long nn = g.n;
                    const unsigned long long passes = (cnt + gridDim.x * DTPB - 1u) / (gridDim.x * DTPB);
                    const unsigned long long ex_max =
                        cnt + (unsigned long long)(g.bfs_block_levels - 1) * (DTPB * 4u) * gridDim.x * passes;
                    bfs_step_levels_body(g, L, cnt, first, s_buf, DTPB * 8, s_m, bfs_visits,
                                         g.bfs_block_levels, 4ull * ex_max <= nn, exact);
                    exact = false;
                } else {
                    const unsigned long long nn = g.n;
                    const int hops = (g.bfs_hops > 1 && cnt <= g.bfs_chain_max &&
                                      4ull * (unsigned long long)g.bfs_hops * cnt <= nn)
                                         ? g.bfs_hops : 1;
                    const bool propagate = 4ull * (unsigned long long)hops * cnt <= nn;
                    bfs_step_body(g, L, cnt, first, s_buf, DTPB * 8, s_m, bfs_visits, hops, propagate,
                                  exact);
                    if (hops > 1) exact = false;
                }
                if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
                if (lead) {
                    const int c = cnt <= 1024u ? 0 : (cnt <= 16384u ? 1 : 2);
                    s_step_ns[c] += gtimer() - t_step;
                    ++s_step_cnt[c];
                }
                ++L;
                ++levels_total;
                if (L > g.n + 2u) {   // a BFS labels a new node per level
                    if (lead) raise_error(ctl, (int)GPUPR_ERR_INVARIANT);
                    ok = false;
                    break;
                }
            }
            if (!ok) break;
            ++relabels;
            lap(0);
            active_sweep_body(g, s_buf, s_buf + DTPB * 4, s_m);
            if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
            lap(1);
            if (vload(&ctl->act_cnt[0]) == 0u) break;   // maximum preflow
            if (g.nseg) retire_graphs(g);
            // ---- discharge rounds ----
            uint32_t r = 0;
            unsigned long long visits = 0;
            unsigned long long budget = p.budget;
            for (;;) {
                const uint32_t first = prefetch_entry((r & 1) ? g.act[1] : g.act[0], g.n);
                const uint32_t cnt = min(vload(&ctl->act_cnt[r % 3]), g.n);
                if (cnt == 0) break;
                if (rounds_total >= p.max_rounds) {
                    if (lead) raise_error(ctl, (int)GPUPR_ERR_MAX_ROUNDS);
                    ok = false;
                    break;
                }
                if (lead) ctl->act_cnt[(r + 2) % 3] = 0u;
                if (lead) s_dr_t0 = gtimer();   // shared: keeps the discharge's registers free
                discharge_body<kAgg>(g, r, cnt, first, s_buf, DTPB * 8, s_m, w);
                if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
                if (lead) {
                    const int c = cnt <= 4096u ? 0 : (cnt <= 131072u ? 1 : 2);
                    s_dr_ns[c] += gtimer() - s_dr_t0;
                    ++s_dr_cnt[c];
                }
                ++r;
                ++rounds_total;
                visits += cnt;
                if (g.nseg && r == 1u && budget) {
                    // the work between relabels follows the nodes still being
                    // solved (read after a barrier that follows every
                    // retirement of this relabel, so all blocks agree)
                    const unsigned long long live = (unsigned long long)g.n - vload(&ctl->retired_nodes);
                    budget = (unsigned long long)((double)p.budget * ((double)live / (double)g.n)) + 1ull;
                }
                if (p.relabel_rounds && r >= p.relabel_rounds) break;
                if (budget && visits > budget) break;
            }
            if (!ok) break;
            if (lead) {
                for (int k = 0; k < 3; ++k) {
                    ctl->act_cnt[k] = 0u;
                    ctl->bfs_cnt[k] = 0u;
                    ctl->lab_cnt[k] = 0u;
                    ctl->bu_cnt[k] = 0u;
                }
                // the reached set of this relabel: the next one's candidates
                ctl->cand_cnt = ctl->cand_build;
                ctl->bu_cnt[0] = ctl->cand_build;
                ctl->cand_build = 0u;
            }
            if (!(ok = grid_barrier(ctl, bar_target, deadline, p.wait_ns, &s_ok))) break;
            lap(2);
        }
        if (lead) {
            ctl->rounds_done = (uint32_t)rounds_total;
            ctl->bfs_levels = levels_total;
            ctl->relabel_phases = relabels;
            for (int k = 0; k < 3; ++k) {
                ctl->step_cnt[k] = s_step_cnt[k];
                ctl->step_ns[k] = s_step_ns[k];
                ctl->dround_cnt[k] = s_dr_cnt[k];
                ctl->dround_ns[k] = s_dr_ns[k];
            }
            ctl->bfs_ns = s_clk[0];
            ctl->sweep_ns = s_clk[1];
            ctl->discharge_ns = s_clk[2];
            ctl->tile_steps = tsteps;
        }
    }
    reduce_work(ctl, w, bfs_visits, s_red);
    if (kTiles) {
        const unsigned long long x = warp_block_sum(twrites, s_red);
        if (threadIdx.x == 0) {
            if (x) atomicAdd(&ctl->tile_writes, x);
            if (tlevels) atomicAdd(&ctl->bfs_visits, tlevels);   // levels run inside tiles
            if (tprocs) atomicAdd(&ctl->tile_procs, tprocs);
            if (tloads) atomicAdd(&ctl->tile_loads, tloads);
        }
    }
}

// First graph of every sweep chunk: the largest k with off[k] <= the chunk's
// first node.
__global__ void __launch_bounds__(DTPB) k_chunk_seg(uint32_t nchunks, uint32_t nseg,
                                                    const uint32_t* __restrict__ off,
                                                    uint32_t* __restrict__ chunk_seg)
{
    for (uint32_t c = blockIdx.x * DTPB + threadIdx.x; c < nchunks; c += gridDim.x * DTPB) {
        const uint32_t v0 = c * SWEEP_CHUNK;
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(off + mid) <= v0) lo = mid;
            else hi = mid;
        }
        chunk_seg[c] = lo;
    }
}

__global__ void __launch_bounds__(DTPB) k_prepare_raw(uint32_t n, const int4* __restrict__ nbr,
                                                      const uint4* __restrict__ cap,
                                                      const uint32_t* __restrict__ src,
                                                      const uint32_t* __restrict__ snk,
                                                      uint4* __restrict__ res,
                                                      int32_t* __restrict__ term,
                                                      unsigned long long* base, int32_t* err)
{
    __shared__ unsigned long long s_red[DTPB / 32];
    unsigned long long b = 0;
    for (uint32_t v = blockIdx.x * DTPB + threadIdx.x; v < n; v += gridDim.x * DTPB) {
        const int4 nb = __ldg(nbr + v);
        uint4 c = __ldg(cap + v);
        if (nb.x < 0) c.x = 0;
        if (nb.y < 0) c.y = 0;
        if (nb.z < 0) c.z = 0;
        if (nb.w < 0) c.w = 0;
        if (c.x > 0x7FFFFFFFu || c.y > 0x7FFFFFFFu || c.z > 0x7FFFFFFFu || c.w > 0x7FFFFFFFu)
            atomicExch(err, 1);
        res[v] = c;
        const long long s = __ldg(src + v), k = __ldg(snk + v);
        const long long d = s - k;
        if (d < -2147483647LL || d > 2147483647LL) atomicExch(err, 1);
        term[v] = (int32_t)d;
        b += (unsigned long long)(s < k ? s : k);
    }
    const unsigned long long x = warp_block_sum(b, s_red);
    if (threadIdx.x == 0 && x) atomicAdd(base, x);
}

__global__ void k_bounded_wait(const volatile uint32_t* flag, unsigned long long limit_ns,
                               int32_t* status)
{
    unsigned long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;) {
        if (*flag != 0u) { *status = 0; return; }
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) { *status = (int32_t)GPUPR_ERR_TIMEOUT; return; }
        __nanosleep(1000);
    }
}

Ctl& read_ctl(Ctl* h, const Ctl* d, cudaStream_t s)
{
    GPUPR_CUDA(cudaMemcpyAsync(h, d, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (h->error)
        throw Error{(gpupr_status)h->error,
                    "GPUPr-B200 device invariant failed code=" + std::to_string(h->error)};
    return *h;
}

}  // namespace

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    GPUPR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int v = 0;
        GPUPR_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        cached[dev] = v > 0 ? v : 1;
    }
    return cached[dev];
}

SolveOptions resolve_options(const gpupr_solve_options* o, int local_steps_raw, int period_raw,
                             uint64_t max_rounds_raw)
{
    SolveOptions r;
    int ls = local_steps_raw;
    int period = period_raw;
    uint64_t mr = max_rounds_raw;
    if (o) {
        if (o->local_steps) ls = o->local_steps;
        if (o->global_relabel_period) period = o->global_relabel_period;
        if (o->max_rounds) mr = o->max_rounds;
        if (o->time_limit_seconds > 0) r.time_limit_s = o->time_limit_seconds;
        if (o->round_batch > 0) r.round_batch = o->round_batch;
        if (o->bfs_batch > 0) r.bfs_batch = o->bfs_batch;
        if (o->block_size > 0) r.block = o->block_size;
        if (o->blocks_per_sm > 0) r.blocks_per_sm = o->blocks_per_sm;
        if (o->work_relabel_factor > 0) r.work_factor = o->work_relabel_factor;
        r.engine = o->engine;
        if (o->chain_hops > 0) r.chain_hops = o->chain_hops;
        if (o->chain_max_active > 0) r.chain_max_active = o->chain_max_active;
        if (o->bfs_chain_hops > 0) r.bfs_chain_hops = o->bfs_chain_hops;
        r.bfs_tail_max = o->bfs_tail_max;
        r.discharge_warp_aggregate = o->discharge_warp_aggregate;
        if (o->bfs_chain_max_frontier > 0) r.bfs_chain_max_frontier = o->bfs_chain_max_frontier;
        r.bfs_bottom_up = o->bfs_bottom_up;
        r.relabel_tiles = o->relabel_tiles;
        r.bfs_block_levels = o->bfs_block_levels;
        r.bfs_in_arc_masks = o->bfs_in_arc_masks;
        if (o->bfs_bottom_up_ratio > 0) r.bfs_bottom_up_ratio = o->bfs_bottom_up_ratio;
    }
    // clamps of gpu_push_relabel_fast.cu:421-424 and :476-480
    if (ls < 1) ls = 1;
    if (ls > 32) ls = 32;
    if (period < 0) period = 0;
    if (!mr) mr = 2000000ull;
    r.local_steps = ls;
    r.relabel_rounds = period > 0 ? ((period + ls - 1) / ls < 1 ? 1 : (period + ls - 1) / ls) : 0;
    r.period = period;
    r.max_rounds = mr;
    return r;
}

int persistent_blocks_per_sm()
{
    int bps = 0;
    GPUPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_solve_persistent<false, false>, DTPB, 0));
    return bps;
}

bool use_persistent_engine(const SolveOptions& opt)
{
    if (opt.engine == 1) return false;
    int dev = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return coop != 0;
}

// The whole solve as one cooperative launch of k_solve_persistent.
void solve_persistent(const SolveView& g, const SolveOptions& opt, cudaStream_t s, SolveResult& out)
{
    using Clock = std::chrono::steady_clock;
    int bps = 0;
    const bool agg = opt.discharge_warp_aggregate > 0;
    const void* kern = g.arcm ? (agg ? (const void*)k_solve_persistent<true, true>
                                     : (const void*)k_solve_persistent<false, true>)
                              : (agg ? (const void*)k_solve_persistent<true, false>
                                     : (const void*)k_solve_persistent<false, false>);
    const size_t dsmem = g.arcm ? TILE_SMEM : 0u;
    if (dsmem) GPUPR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    GPUPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, DTPB, dsmem));
    if (bps < 1) throw Error{GPUPR_ERR_CUDA, "persistent solver kernel cannot be resident"};
    // resident blocks per SM: a step of a small graph is one chain of
    // dependent L2 round trips plus a grid barrier whose cost grows with the
    // number of blocks, while a large graph needs the threads to cover its
    // frontiers and its blocks' BFS sub-levels.  Measured on B200 with the
    // default BFS steps (15 graphs of 0.24-7.4M free nodes, three generators
    // and the config-1 Delaunay proxy, median of 7): 2 is best or within 3%
    // below 1.5M free nodes, 3 up to ~5M, 4 above (config 1: 3.3 ms at 2,
    // 1.20 at 3; a 5.6M-node torus 5.07 at 3, 4.87 at 4).
    // An autotuned entry for this size class replaces the rule.
    TuneEntry te;
    const bool tuned = tune_lookup(g.n, &te);
    const int want = opt.blocks_per_sm > 0 ? opt.blocks_per_sm
                     : tuned                ? te.blocks_per_sm
                     : g.n < 1500000u       ? 2
                     : g.n < 5000000u       ? 3
                                            : 4;
    int used = want < bps ? want : bps;
    if (opt.max_blocks_per_sm > 0 && used > opt.max_blocks_per_sm) used = opt.max_blocks_per_sm;
    const unsigned grid = (unsigned)(sm_count() * used);
    PersistParams p{};
    p.max_rounds = opt.max_rounds;
    // Global relabels: a discharge phase ends once its node visits exceed
    // work_factor x n (measured on B200: 2 suits graphs below ~500k free
    // nodes, 1 up to ~10M, 0.5 above: 19M nodes 14.5 vs 16.6 ms, a 64-graph
    // union of 50M 80.7 vs 89.8 ms), or after global_relabel_period rounds, a
    // cap the work rule normally reaches first.  The result does not depend on this
    // schedule: the solve always ends with an exact relabel.
    p.relabel_rounds = (uint32_t)(opt.period > 0 ? opt.period : 0);
    const double wf = opt.work_factor > 0 ? opt.work_factor
                      : tuned                ? te.work_factor
                      : g.n < 500000u        ? 2.0
                      : g.n < 10000000u      ? 1.0
                                             : 0.5;
    const double budget = wf * (double)g.n;
    p.budget = budget > 1.8e19 ? 0ull : (unsigned long long)budget;
    p.limit_ns = (unsigned long long)(opt.time_limit_s * 1e9);
    p.wait_ns = 10ull * 1000ull * 1000ull * 1000ull;   // one step never takes this long

    Ctl* pc = pinned_ctl();
    cudaEvent_t e0 = timing_event(2), e1 = timing_event(3);
    const auto t0 = Clock::now();
    GPUPR_CUDA(cudaMemsetAsync(g.ctl, 0, sizeof(Ctl), s));
    GPUPR_CUDA(cudaEventRecord(e0, s));
    SolveView gv = g;
    // Chained discharge pays where a round is a latency chain (few active
    // nodes) and can multiply node visits in wide rounds.  Measured on B200
    // with 4 hops over 18 graphs below 1.5M free nodes: chaining in rounds of
    // up to 131072 active nodes took 59.5 ms in all against 69.8 ms with
    // 4096; between 1.5M and 2M, 32768 was best; above, only 4096 did not
    // slow any graph down (a 2.9M-node torus: 6.6 ms, 10.0 with 32768).  The
    // autotuner may pick another setting.
    gv.chain_hops = opt.chain_hops > 0 ? opt.chain_hops : tuned ? te.chain_hops : 4;
    gv.bfs_hops = opt.bfs_chain_hops > 0 ? std::min(opt.bfs_chain_hops, 64) : BFS_CHAIN_HOPS;
    // BFS steps expand BFS_BLOCK_LEVELS levels per block by default (measured
    // against per-thread chains of 4: benchmark graph 77.7 -> 68.0 ms, 8M-tet
    // open box 14.1 -> 12.5 ms, 3M-tet torus 2.27 -> 1.98 ms; 8 and 32 levels
    // within 1-3% of 16); 1 keeps the chains
    gv.bfs_block_levels = opt.bfs_block_levels == 1 ? 0
                          : opt.bfs_block_levels > 1 ? std::min(opt.bfs_block_levels, 64)
                                                     : BFS_BLOCK_LEVELS;
    gv.warp_agg = agg ? 1 : 0;
    // BFS steps chain over frontiers of any size the queue bound allows
    // (measured against a 65,536-node limit: benchmark graph 78.3 -> 77.2 ms,
    // 3M-tet torus 2.30 -> 2.28 ms, 8M-tet open box 14.5 -> 14.0 ms)
    gv.bfs_chain_max = opt.bfs_chain_max_frontier > 0 ? (uint32_t)opt.bfs_chain_max_frontier
                                                      : 0xFFFFFFFFu;
    gv.tail_max = opt.bfs_tail_max < 0 ? 0u
                  : opt.bfs_tail_max > 0 ? std::min<uint32_t>((uint32_t)opt.bfs_tail_max, TAIL_CAP)
                                         : BFS_TAIL_DEFAULT;
    gv.chain_max_active = opt.chain_max_active > 0 ? (uint32_t)opt.chain_max_active
                          : tuned                  ? (uint32_t)te.chain_max_active
                          : g.n < 1500000u         ? 131072u
                          : g.n < 2000000u         ? 32768u
                                                   : 4096u;
    void* args[] = {&gv, &p};
    GPUPR_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(DTPB), args, dsmem, s));
    GPUPR_CUDA(cudaEventRecord(e1, s));
    GPUPR_CUDA(cudaMemcpyAsync(pc, g.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    const Ctl& hc = *pc;
    if (hc.error == (int)GPUPR_ERR_TIMEOUT)
        throw Error{GPUPR_ERR_TIMEOUT, "GPUPr-FAST-v6.30 solve exceeded 240s safety limit"};
    if (hc.error == (int)GPUPR_ERR_MAX_ROUNDS)
        throw Error{GPUPR_ERR_MAX_ROUNDS, "GPUPr-FAST-v6.30 max macro rounds exceeded"};
    if (hc.error)
        throw Error{(gpupr_status)hc.error,
                    "GPUPr-B200 device invariant failed code=" + std::to_string(hc.error)};
    float ms = 0.f;
    GPUPR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    out.engine = 2;
    out.blocks_per_sm = used;
    out.work_factor = wf;
    out.chain_hops = gv.chain_hops;
    out.chain_max_active = (int)gv.chain_max_active;
    out.launches = 1;
    out.raw_flow = (int64_t)hc.sink_flow;
    out.rounds = hc.rounds_done;
    out.relabels = hc.relabel_phases;
    out.node_visits = hc.node_visits;
    out.pushes = hc.pushes;
    out.bfs_visits = hc.bfs_visits;
    out.bfs_levels = hc.bfs_levels;
    out.solve_device_ms = ms;
    out.discharge_launches = 1;
    // phase split from block 0's clock; the active sweeps count as relabel work
    out.bfs_ms = (double)(hc.bfs_ns + hc.sweep_ns) * 1e-6;
    out.discharge_ms = (double)hc.discharge_ns * 1e-6;
    out.sweep_ms = (double)hc.sweep_ns * 1e-6;
    out.graphs_retired = hc.segs_retired;
    out.bottom_up_steps = hc.bu_steps;
    out.tail_steps = hc.tail_steps;
    out.tail_levels = hc.tail_levels;
    out.relabel_tiles = g.arcm ? 1 : 0;
    out.tile_steps = hc.tile_steps;
    out.tile_procs = hc.tile_procs;
    out.tile_loads = hc.tile_loads;
    out.tile_writes = hc.tile_writes;
    for (int k = 0; k < 3; ++k) {
        out.step_cnt[k] = hc.step_cnt[k];
        out.step_ms[k] = (double)hc.step_ns[k] * 1e-6;
        out.dround_cnt[k] = hc.dround_cnt[k];
        out.dround_ms[k] = (double)hc.dround_ns[k] * 1e-6;
    }
    out.solve_s = std::chrono::duration<double>(Clock::now() - t0).count();
}

void solve_push_relabel(uint32_t n, const int4* d_nbr, uint32_t* d_res, const uint8_t* d_rev,
                        const uint32_t* d_pair, int32_t* d_term, SolveWorkspace& w,
                        const SolveOptions& opt, cudaStream_t s, SolveResult& out,
                        const Segments* segments)
{
    using Clock = std::chrono::steady_clock;
    out = SolveResult{};
    if (!n) return;
    if (w.excess.n < n) {
        w.excess = DevBuf<long long>(n, s);
        w.height = DevBuf<uint32_t>(n, s);
        w.q0 = DevBuf<uint32_t>(n, s);
        w.q1 = DevBuf<uint32_t>(n, s);
        w.q2 = DevBuf<uint32_t>(n, s);
    }
    if (!w.ctl.p) w.ctl = DevBuf<Ctl>(1, s);
    out.workspace_bytes = w.bytes();

    SolveView g{};
    g.n = n;
    g.nbr = d_nbr;
    g.res = d_res;
    g.rev = d_rev;
    g.pair = reinterpret_cast<const uint4*>(d_pair);
    g.term = d_term;
    g.excess = w.excess.p;
    g.height = w.height.p;
    g.act[0] = w.q0.p;
    g.act[1] = w.q1.p;
    g.fr[0] = w.q2.p;
    g.fr[1] = w.q1.p;   // act[1] is idle while a BFS runs
    g.ctl = w.ctl.p;
    g.local_steps = opt.local_steps;

    if (use_persistent_engine(opt)) {
        if (segments && segments->nseg > 1u && segments->d_off) {
            const uint32_t nseg = segments->nseg;
            const uint32_t nchunks = (n + SWEEP_CHUNK - 1u) / SWEEP_CHUNK;
            if (w.chunk_seg.n < nchunks) w.chunk_seg = DevBuf<uint32_t>(nchunks, s);
            if (w.seg_live.n < nseg) {
                w.seg_live = DevBuf<uint32_t>(nseg, s);
                w.seg_act = DevBuf<uint32_t>(nseg, s);
            }
            GPUPR_CUDA(cudaMemsetAsync(w.seg_live.p, 0x01, (size_t)nseg * 4u, s));   // all live
            GPUPR_CUDA(cudaMemsetAsync(w.seg_act.p, 0, (size_t)nseg * 4u, s));
            const unsigned cg = (unsigned)std::min<uint32_t>((nchunks + DTPB - 1u) / DTPB,
                                                             (uint32_t)sm_count() * 8u);
            k_chunk_seg<<<cg, DTPB, 0, s>>>(nchunks, nseg, segments->d_off, w.chunk_seg.p);
            GPUPR_CUDA(cudaGetLastError());
            out.launches += 1;
            g.nseg = nseg;
            g.seg_off = segments->d_off;
            g.chunk_seg = w.chunk_seg.p;
            g.seg_live = w.seg_live.p;
            g.seg_act = w.seg_act.p;
            out.workspace_bytes = w.bytes();
        }
        const bool tiles = opt.relabel_tiles > 0 ||
                           (opt.relabel_tiles == 0 && n >= RELABEL_TILES_DEFAULT_MIN);
        if (tiles) {
            const uint32_t nt = (uint32_t)(((uint64_t)n + RELABEL_TILE - 1u) >> RELABEL_TILE_SHIFT);
            if (w.arcm.n < n) w.arcm = DevBuf<uint8_t>(n, s);
            if (w.tile_stamp.n < nt) w.tile_stamp = DevBuf<uint32_t>(nt, s);
            GPUPR_CUDA(cudaMemsetAsync(w.tile_stamp.p, 0, (size_t)nt * 4u, s));
            g.arcm = w.arcm.p;
            g.tile_stamp = w.tile_stamp.p;
            g.ntiles = nt;
        } else if (opt.bfs_in_arc_masks > 0 || (opt.bfs_in_arc_masks == 0 && BFS_IN_ARC_MASKS_DEFAULT)) {
            if (w.inm.n < n) w.inm = DevBuf<uint8_t>(n, s);
            g.inm = w.inm.p;
        } else {
            if (w.inrow.n < n) w.inrow = DevBuf<int4>(n, s);
            g.inrow = w.inrow.p;
        }
        out.workspace_bytes = w.bytes();
        if (opt.bfs_bottom_up && !tiles) {
            if (w.cand0.n < n) {
                w.cand0 = DevBuf<uint32_t>(n, s);
                w.cand1 = DevBuf<uint32_t>(n, s);
            }
            g.cand[0] = w.cand0.p;
            g.cand[1] = w.cand1.p;
            g.bottom_up = 1;
            g.bu_ratio = (float)(opt.bfs_bottom_up_ratio > 0 ? opt.bfs_bottom_up_ratio : 1.0);
            out.workspace_bytes = w.bytes();
        }
        const uint64_t pre = out.launches;
        solve_persistent(g, opt, s, out);
        out.launches += pre;
        return;
    }
    out.engine = 1;
    const double engine1_wf = opt.work_factor > 0 ? opt.work_factor : 3.0;
    const int grid = sm_count() * (opt.blocks_per_sm > 0 ? opt.blocks_per_sm : 4);
    Ctl* pc = pinned_ctl();
    cudaEvent_t e0 = timing_event(2), e1 = timing_event(3), ba = timing_event(4), bb = timing_event(5);
    // device time of one batch (the host waits for the batch anyway)
    auto batch_ms = [&]() {
        float ms = 0.f;
        GPUPR_CUDA(cudaEventElapsedTime(&ms, ba, bb));
        return (double)ms;
    };

    GPUPR_CUDA(cudaMemsetAsync(w.ctl.p, 0, sizeof(Ctl), s));
    GPUPR_CUDA(cudaEventRecord(e0, s));
    k_init_excess<<<grid, DTPB, 0, s>>>(n, d_term, w.excess.p);
    GPUPR_CUDA(cudaGetLastError());
    out.launches += 1;

    const auto t0 = Clock::now();
    uint64_t rounds_total = 0;
    double last_bfs_s = 0.0;
    for (;;) {
        // ---- exact global relabel: backward BFS from the sink ----
        const auto b0 = Clock::now();
        GPUPR_CUDA(cudaMemsetAsync(w.ctl.p, 0, offsetof(Ctl, error), s));
        GPUPR_CUDA(cudaEventRecord(ba, s));
        k_bfs_seed<<<grid, DTPB, 0, s>>>(g);
        GPUPR_CUDA(cudaGetLastError());
        out.launches += 1;
        out.bfs_launches += 1;
        uint32_t L = 1;
        for (;;) {
            for (int b = 0; b < opt.bfs_batch; ++b, ++L) {
                k_bfs_level<<<grid, DTPB, 0, s>>>(g, L);
                GPUPR_CUDA(cudaGetLastError());
            }
            GPUPR_CUDA(cudaEventRecord(bb, s));
            out.launches += (uint64_t)opt.bfs_batch;
            out.bfs_launches += (uint64_t)opt.bfs_batch;
            const Ctl& hc = read_ctl(pc, w.ctl.p, s);
            out.bfs_ms += batch_ms();
            GPUPR_CUDA(cudaEventRecord(ba, s));
            if (hc.bfs_done) break;
            if ((uint64_t)L > (uint64_t)n + 2u)
                throw Error{GPUPR_ERR_INVARIANT, "GPUPr-FAST-v6.30 BFS exceeded n+1 levels"};
        }
        ++out.relabels;
        out.bfs_levels += pc->bfs_levels;
        last_bfs_s = std::chrono::duration<double>(Clock::now() - b0).count();
        const uint32_t active = pc->act_cnt[0];
        if (active == 0) break;   // maximum preflow: no excess can reach the sink
        if (rounds_total >= opt.max_rounds)
            throw Error{GPUPR_ERR_MAX_ROUNDS, "GPUPr-FAST-v6.30 max macro rounds exceeded"};

        // ---- discharge rounds until idle, period or work budget ----
        const unsigned long long visits0 = pc->node_visits;
        uint32_t r = 0;
        for (;;) {
            uint64_t left = opt.max_rounds - rounds_total;
            int batch = opt.round_batch;
            if ((uint64_t)batch > left) batch = (int)left;
            GPUPR_CUDA(cudaEventRecord(ba, s));
            for (int b = 0; b < batch; ++b, ++r) {
                k_discharge<<<grid, DTPB, 0, s>>>(g, r);
                GPUPR_CUDA(cudaGetLastError());
            }
            GPUPR_CUDA(cudaEventRecord(bb, s));
            out.launches += (uint64_t)batch;
            out.discharge_launches += (uint64_t)batch;
            const Ctl& hc = read_ctl(pc, w.ctl.p, s);
            out.discharge_ms += batch_ms();
            rounds_total = hc.rounds_done;
            const bool idle = hc.act_cnt[r % 3] == 0u;
            if (idle) break;
            if (rounds_total >= opt.max_rounds)
                throw Error{GPUPR_ERR_MAX_ROUNDS, "GPUPr-FAST-v6.30 max macro rounds exceeded"};
            if (opt.relabel_rounds > 0 && r >= (uint32_t)opt.relabel_rounds) break;
            if ((double)(hc.node_visits - visits0) > engine1_wf * (double)n)
                break;
            const double el = std::chrono::duration<double>(Clock::now() - t0).count();
            if (el > opt.time_limit_s)
                throw Error{GPUPR_ERR_TIMEOUT, "GPUPr-FAST-v6.30 solve exceeded 240s safety limit"};
        }
    }
    GPUPR_CUDA(cudaEventRecord(e1, s));
    GPUPR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    GPUPR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const Ctl& hc = *pc;
    out.raw_flow = (int64_t)hc.sink_flow;
    out.rounds = hc.rounds_done;
    out.node_visits = hc.node_visits;
    out.pushes = hc.pushes;
    out.bfs_visits = hc.bfs_visits;
    out.solve_device_ms = ms;
    out.final_relabel_s = last_bfs_s;
    out.solve_s = std::chrono::duration<double>(Clock::now() - t0).count();
}

int64_t prepare_raw_graph(uint32_t n, const uint32_t* d_cap, const uint32_t* d_src,
                          const uint32_t* d_snk, const int32_t* d_nbr, uint32_t* d_res,
                          int32_t* d_term, cudaStream_t s, uint64_t* launches)
{
    DevBuf<unsigned long long> base(1, s);
    DevBuf<int32_t> err(1, s);
    GPUPR_CUDA(cudaMemsetAsync(base.p, 0, sizeof(unsigned long long), s));
    GPUPR_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t), s));
    const int grid = sm_count() * 8;
    k_prepare_raw<<<grid, DTPB, 0, s>>>(n, reinterpret_cast<const int4*>(d_nbr),
                                        reinterpret_cast<const uint4*>(d_cap), d_src, d_snk,
                                        reinterpret_cast<uint4*>(d_res), d_term, base.p, err.p);
    GPUPR_CUDA(cudaGetLastError());
    *launches += 1;
    unsigned long long hb = 0;
    int32_t he = 0;
    GPUPR_CUDA(cudaMemcpyAsync(&hb, base.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaMemcpyAsync(&he, err.p, sizeof(he), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (he) throw Error{GPUPR_ERR_BUILD, "capacity or terminal outside the int32 range"};
    return (int64_t)hb;
}

gpupr_status bounded_wait_selftest(uint32_t limit_us, cudaStream_t s)
{
    DevBuf<uint32_t> flag(1, s);
    DevBuf<int32_t> st(1, s);
    GPUPR_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(uint32_t), s));
    GPUPR_CUDA(cudaMemsetAsync(st.p, 0xFF, sizeof(int32_t), s));
    k_bounded_wait<<<1, 1, 0, s>>>(flag.p, (unsigned long long)limit_us * 1000ull, st.p);
    GPUPR_CUDA(cudaGetLastError());
    int32_t h = -1;
    GPUPR_CUDA(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    return (gpupr_status)h;
}

}  // namespace gpupr

namespace gpupr {

// ---------------------------------------------------------------------------
// Allocation-free solve: scratch in a static device array.
//
// For callers that cannot allocate device memory (a host application that owns
// the whole device heap through its own allocator, or a caller that must not
// call the CUDA allocator mid-pipeline): every buffer the solver needs beyond
// the caller's graph and output lives in g_noalloc_scratch below.  The array is
// part of every context that loads this library, for the lifetime of the
// process.  It is shared by all calls: two calls whose work overlaps on the GPU
// (different streams or threads at the same time) corrupt each other.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t NA_ALIGN = 256;
constexpr size_t na_round(size_t b) { return (b + NA_ALIGN - 1) / NA_ALIGN * NA_ALIGN; }
// layout: control block | error flag | excess | height | 3 queues | reverse
// slots | arc-pair residual sums
constexpr size_t NA_CTL = 0;
constexpr size_t NA_ERR = na_round(sizeof(Ctl));
constexpr size_t NA_EXCESS = NA_ERR + NA_ALIGN;
constexpr size_t NA_HEIGHT = NA_EXCESS + na_round((size_t)NOALLOC_MAX_NODES * 8u);
constexpr size_t NA_Q0 = NA_HEIGHT + na_round((size_t)NOALLOC_MAX_NODES * 4u);
constexpr size_t NA_Q1 = NA_Q0 + na_round((size_t)NOALLOC_MAX_NODES * 4u);
constexpr size_t NA_Q2 = NA_Q1 + na_round((size_t)NOALLOC_MAX_NODES * 4u);
constexpr size_t NA_REV = NA_Q2 + na_round((size_t)NOALLOC_MAX_NODES * 4u);
constexpr size_t NA_PAIR = NA_REV + na_round((size_t)NOALLOC_MAX_NODES);
constexpr size_t NA_BYTES = NA_PAIR + na_round((size_t)NOALLOC_MAX_NODES * 16u);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

std::mutex g_na_mu;
unsigned char* g_na_ptr[64] = {};

// Device address of the scratch array on the current device.  The host-side
// name g_noalloc_scratch is only a stand-in for the symbol, so the address is
// looked up once per device (with that device current) and cached; `refresh`
// looks it up again (after cudaDeviceReset the module, and with it the array,
// is loaded anew and may sit elsewhere).  The lookup loads this file's device
// module if it is not loaded yet (CUDA loads modules lazily by default), which
// is when the array's memory is committed on the device.
unsigned char* noalloc_scratch(bool refresh)
{
    int dev = 0;
    GPUPR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "device ordinal out of range"};
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev] || refresh) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            g_na_ptr[dev] = nullptr;
            throw Error{e == cudaErrorMemoryAllocation ? GPUPR_ERR_OUT_OF_MEMORY : GPUPR_ERR_CUDA,
                        std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                            cudaGetErrorString(e)};
        }
        g_na_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_na_ptr[dev];
}

// Host copy of the control block without pinned memory: a pageable
// cudaMemcpyAsync on the stream, then a stream synchronize.
const Ctl& read_ctl_stack(Ctl& h, const Ctl* d, cudaStream_t s)
{
    GPUPR_CUDA(cudaMemcpyAsync(&h, d, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    if (h.error)
        throw Error{(gpupr_status)h.error, "GPUPr-B200 device invariant failed"};
    return h;
}

}  // namespace

uint64_t noalloc_prepare()
{
    noalloc_scratch(true);
    return (uint64_t)NA_BYTES;
}

void solve_reduced_noalloc(uint32_t n, int32_t* d_nbr, uint32_t* d_res, int32_t* d_term,
                           uint8_t* d_partition, const SolveOptions& opt, cudaStream_t s,
                           SolveResult& out)
{
    using Clock = std::chrono::steady_clock;
    out = SolveResult{};
    if (!n) return;
    if (n > NOALLOC_MAX_NODES)
        throw Error{GPUPR_ERR_INVALID_ARGUMENT,
                    "gpupr_solve_reduced_noalloc: n exceeds the static scratch limit of 1048576 nodes"};
    unsigned char* base = noalloc_scratch(false);
    Ctl* ctl = reinterpret_cast<Ctl*>(base + NA_CTL);
    int32_t* err = reinterpret_cast<int32_t*>(base + NA_ERR);
    uint8_t* rev = base + NA_REV;
    uint32_t* pair = reinterpret_cast<uint32_t*>(base + NA_PAIR);
    const int4* nbr = reinterpret_cast<const int4*>(d_nbr);
    compute_reverse_slots_noalloc(n, nbr, d_res, rev, pair, err, s);
    out.launches += 1;

    SolveView g{};
    g.n = n;
    g.nbr = nbr;
    g.res = d_res;
    g.rev = rev;
    g.pair = reinterpret_cast<const uint4*>(pair);
    g.term = d_term;
    g.excess = reinterpret_cast<long long*>(base + NA_EXCESS);
    g.height = reinterpret_cast<uint32_t*>(base + NA_HEIGHT);
    g.act[0] = reinterpret_cast<uint32_t*>(base + NA_Q0);
    g.act[1] = reinterpret_cast<uint32_t*>(base + NA_Q1);
    g.fr[0] = reinterpret_cast<uint32_t*>(base + NA_Q2);
    g.fr[1] = g.act[1];
    g.ctl = ctl;
    g.local_steps = opt.local_steps;
    const int grid = sm_count() * (opt.blocks_per_sm > 0 ? opt.blocks_per_sm : 4);
    const double engine1_wf = opt.work_factor > 0 ? opt.work_factor : 3.0;

    Ctl hc{};
    // the array keeps the previous call's contents: the control block must
    // start at zero; every other buffer is written before it is read
    GPUPR_CUDA(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
    k_init_excess<<<grid, DTPB, 0, s>>>(n, d_term, g.excess);
    GPUPR_CUDA(cudaGetLastError());
    out.launches += 1;
    const auto t0 = Clock::now();
    uint64_t rounds_total = 0;
    for (;;) {
        GPUPR_CUDA(cudaMemsetAsync(ctl, 0, offsetof(Ctl, error), s));
        k_bfs_seed<<<grid, DTPB, 0, s>>>(g);
        GPUPR_CUDA(cudaGetLastError());
        out.launches += 1;
        uint32_t L = 1;
        for (;;) {
            for (int b = 0; b < opt.bfs_batch; ++b, ++L) {
                k_bfs_level<<<grid, DTPB, 0, s>>>(g, L);
                GPUPR_CUDA(cudaGetLastError());
            }
            out.launches += (uint64_t)opt.bfs_batch;
            read_ctl_stack(hc, ctl, s);
            if (hc.bfs_done) break;
            if ((uint64_t)L > (uint64_t)n + 2u)
                throw Error{GPUPR_ERR_INVARIANT, "GPUPr-FAST-v6.30 BFS exceeded n+1 levels"};
        }
        ++out.relabels;
        out.bfs_levels += hc.bfs_levels;
        if (hc.act_cnt[0] == 0) break;
        if (rounds_total >= opt.max_rounds)
            throw Error{GPUPR_ERR_MAX_ROUNDS, "GPUPr-FAST-v6.30 max macro rounds exceeded"};
        const unsigned long long visits0 = hc.node_visits;
        uint32_t r = 0;
        for (;;) {
            const uint64_t left = opt.max_rounds - rounds_total;
            int batch = opt.round_batch;
            if ((uint64_t)batch > left) batch = (int)left;
            for (int b = 0; b < batch; ++b, ++r) {
                k_discharge<<<grid, DTPB, 0, s>>>(g, r);
                GPUPR_CUDA(cudaGetLastError());
            }
            out.launches += (uint64_t)batch;
            read_ctl_stack(hc, ctl, s);
            rounds_total = hc.rounds_done;
            if (hc.act_cnt[r % 3] == 0u) break;
            if (rounds_total >= opt.max_rounds)
                throw Error{GPUPR_ERR_MAX_ROUNDS, "GPUPr-FAST-v6.30 max macro rounds exceeded"};
            if (opt.relabel_rounds > 0 && r >= (uint32_t)opt.relabel_rounds) break;
            if ((double)(hc.node_visits - visits0) > engine1_wf * (double)n)
                break;
            if (std::chrono::duration<double>(Clock::now() - t0).count() > opt.time_limit_s)
                throw Error{GPUPR_ERR_TIMEOUT, "GPUPr-FAST-v6.30 solve exceeded 240s safety limit"};
        }
    }
    partition_from_height(n, g.height, d_partition, s, &out.launches);
    GPUPR_CUDA(cudaStreamSynchronize(s));
    out.raw_flow = (int64_t)hc.sink_flow;
    out.rounds = hc.rounds_done;
    out.node_visits = hc.node_visits;
    out.pushes = hc.pushes;
    out.bfs_visits = hc.bfs_visits;
    out.solve_s = std::chrono::duration<double>(Clock::now() - t0).count();
}

// ---------------------------------------------------------------------------
// Autotuner tables: one entry per size class, shared by the process; one
// table for single graphs (class of the free-node count) and one for batches
// (class of the free nodes per graph).
// ---------------------------------------------------------------------------
namespace {
struct TuneTable {
    std::mutex mu;
    TuneEntry e[33];
    bool valid[33] = {};
};
TuneTable g_tune, g_batch_tune;

bool valid_entry(const TuneEntry& e)
{
    return e.size_class >= 0 && e.size_class <= 32 && e.blocks_per_sm >= 1 && e.blocks_per_sm <= 32 &&
           e.work_factor > 0.0 && e.work_factor < 1e6 && e.chain_hops >= 1 && e.chain_hops <= 64 &&
           e.chain_max_active >= 1;
}

bool table_lookup(TuneTable& t, uint32_t n, TuneEntry* out)
{
    std::lock_guard<std::mutex> lk(t.mu);
    const int k = size_class(n);
    if (!t.valid[k]) return false;
    *out = t.e[k];
    return true;
}

void table_store(TuneTable& t, const TuneEntry& e)
{
    if (!valid_entry(e)) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "invalid tuning entry"};
    std::lock_guard<std::mutex> lk(t.mu);
    t.e[e.size_class] = e;
    t.valid[e.size_class] = true;
}

std::vector<TuneEntry> table_all(TuneTable& t)
{
    std::lock_guard<std::mutex> lk(t.mu);
    std::vector<TuneEntry> v;
    for (int k = 0; k <= 32; ++k)
        if (t.valid[k]) v.push_back(t.e[k]);
    return v;
}

void table_replace(TuneTable& t, const std::vector<TuneEntry>& entries)
{
    for (const TuneEntry& e : entries)
        if (!valid_entry(e)) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "invalid tuning entry"};
    std::lock_guard<std::mutex> lk(t.mu);
    for (int k = 0; k <= 32; ++k) t.valid[k] = false;
    for (const TuneEntry& e : entries) {
        t.e[e.size_class] = e;
        t.valid[e.size_class] = true;
    }
}
}  // namespace

int size_class(uint32_t n)
{
    int k = 0;
    while (k < 31 && (n >> (k + 1)) != 0u) ++k;
    return k;
}

bool tune_lookup(uint32_t n, TuneEntry* out) { return table_lookup(g_tune, n, out); }
void tune_store(const TuneEntry& e) { table_store(g_tune, e); }
std::vector<TuneEntry> tune_all() { return table_all(g_tune); }
void tune_replace(const std::vector<TuneEntry>& entries) { table_replace(g_tune, entries); }

bool batch_tune_lookup(uint64_t mean_free, TuneEntry* out)
{
    return table_lookup(g_batch_tune, (uint32_t)std::min<uint64_t>(mean_free, 0xFFFFFFFFull), out);
}
void batch_tune_store(const TuneEntry& e) { table_store(g_batch_tune, e); }
std::vector<TuneEntry> batch_tune_all() { return table_all(g_batch_tune); }
void batch_tune_replace(const std::vector<TuneEntry>& entries) { table_replace(g_batch_tune, entries); }

}  // namespace gpupr
