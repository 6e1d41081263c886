// capi.cu -- the C ABI of libwtivo_gpupr.so (include/wtivo_gpupr.h).
//
// Host orchestration of the graph_cut_fast path: argument checks with the
// reference's messages (native/gpupr/wtivo_gpupr_bindings.cpp:114-133),
// H2D of host-side vertices/labels, GPU reduced-graph build, solve, label
// scatter (bindings.cpp:357-364), D2H of the result and the stats tuple.
// No exception crosses the ABI: every entry point returns a gpupr_status
// and records the message for gpupr_last_error().
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gpupr_internal.cuh"
#include "wtivo_gpupr.h"

namespace gpupr {

namespace {
thread_local std::string g_last_error;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

cudaMemPool_t device_pool()
{
    int dev = 0;
    GPUPR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "device ordinal out of range"};
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        GPUPR_CUDA(cudaMemPoolCreate(&g_pools[dev], &props));
        // keep freed blocks for the next call: repeated cuts reuse the same
        // footprint without cudaMalloc/cudaFree (gpupr_release_cached_memory
        // trims the pool).
        uint64_t keep = UINT64_MAX;
        GPUPR_CUDA(cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return g_pools[dev];
}

void select_device_for(const void* dptr, const char* what)
{
    cudaPointerAttributes a{};
    cudaError_t e = cudaPointerGetAttributes(&a, dptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, std::string(what) + " must be CUDA tensors"};
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, std::string(what) + " must be CUDA tensors"};
    GPUPR_CUDA(cudaSetDevice(a.device));
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

template <class Fn>
gpupr_status guarded(Fn&& fn)
{
    try {
        fn();
        g_last_error.clear();
        return GPUPR_OK;
    } catch (const Error& e) {
        g_last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return GPUPR_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GPUPR_ERR_CUDA;
    } catch (...) {
        g_last_error = "unknown failure";
        return GPUPR_ERR_CUDA;
    }
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : a(timing_event(0)), b(timing_event(1)), s(st)
    {
        GPUPR_CUDA(cudaEventRecord(a, s));
    }
    double stop_ms()
    {
        GPUPR_CUDA(cudaEventRecord(b, s));
        GPUPR_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        GPUPR_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
};

// Device copies of host inputs (no copy when already on the device).
template <class T>
const T* on_device(const T* p, size_t count, int is_device, DevBuf<T>& keep, cudaStream_t s)
{
    if (is_device || count == 0) return p;
    keep = DevBuf<T>(count, s);
    host_to_device(keep.p, p, count * sizeof(T), s);
    return keep.p;
}

void run_graph_cut(const double* vertices, uint64_t nv, int v_dev, const int32_t* d_tets,
                   const int32_t* d_nbrs, uint64_t N, const uint8_t* labels, int l_dev,
                   double fill_T, int32_t threads, int32_t period, uint64_t max_rounds,
                   int32_t local_steps, const gpupr_solve_options* options, uint8_t* out,
                   int out_dev, cudaStream_t s, gpupr_cut_stats* st)
{
    const auto all0 = std::chrono::steady_clock::now();
    if (!st) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "stats pointer is NULL"};
    std::memset(st, 0, sizeof(*st));
    st->threads = threads < 1 ? 1 : threads;
    st->local_steps = local_steps;
    st->n_full = N;
    if (N > 0xFFFFFFFFull) throw Error{GPUPR_ERR_TOO_MANY_TETS, ">2^32 full tets unsupported"};
    if (N == 0) {
        st->native_total_seconds = seconds_since(all0);
        return;
    }
    if (!d_tets || !d_nbrs) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be CUDA tensors"};
    if (!labels || !out) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "labels size mismatch"};
    if (!vertices && nv) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "vertices must be float64 Nx3"};
    if (!aligned(d_tets, 16) || !aligned(d_nbrs, 16))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be 16-byte aligned"};
    select_device_for(d_tets, "tets/neighbors");

    uint64_t launches = 0;
    const auto b0 = std::chrono::steady_clock::now();
    Timer tb(s);
    DevBuf<uint8_t> dlab;
    DevBuf<double> dver;
    const uint8_t* d_labels = on_device(labels, N, l_dev, dlab, s);
    const double* d_vertices = on_device(vertices, nv * 3u, v_dev, dver, s);
    if (v_dev && vertices && !aligned(vertices, 8))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "vertices must be float64 Nx3"};

    BuildInputs in{d_vertices, nv, d_tets, d_nbrs, d_labels, N, fill_T};
    ReducedGraph g;
    BuildInfo info;
    build_reduced_graph(in, g, info, s, &launches);
    st->build_device_ms = tb.stop_ms();
    st->build_seconds = seconds_since(b0);
    st->full_E = info.full_refs / 2u;
    st->fixed_source = info.fixed_source;
    st->fixed_sink = info.fixed_sink;
    st->free_n = info.free_n;

    if (info.free_n == 0) {   // bindings.cpp:191-196: labels unchanged
        if (out_dev) GPUPR_CUDA(cudaMemcpyAsync(out, d_labels, N, cudaMemcpyDeviceToDevice, s));
        else device_to_host(out, d_labels, N, s);
        GPUPR_CUDA(cudaStreamSynchronize(s));
        st->kernel_launches = launches;
        st->native_total_seconds = seconds_since(all0);
        return;
    }

    const SolveOptions opt = resolve_options(options, local_steps, period, max_rounds);
    SolveWorkspace w;
    SolveResult sr;
    solve_push_relabel(g.n, g.nbr.p, g.res.p, g.rev.p, g.pair.p, g.term.p, w, opt, s, sr);
    launches += sr.launches;

    const auto p0 = std::chrono::steady_clock::now();
    DevBuf<uint8_t> dout;
    uint8_t* d_out = out;
    if (!out_dev) {
        dout = DevBuf<uint8_t>(N, s);
        d_out = dout.p;
    }
    GPUPR_CUDA(cudaMemcpyAsync(d_out, d_labels, N, cudaMemcpyDeviceToDevice, s));
    scatter_partition(g.n, g.free_old.p, w.height.p, d_out, s, &launches);
    if (!out_dev) device_to_host(out, d_out, N, s);
    GPUPR_CUDA(cudaStreamSynchronize(s));
    st->partition_seconds = seconds_since(p0);

    st->raw_flow = sr.raw_flow;
    st->adjusted_flow = sr.raw_flow + info.terminal_base_flow;
    st->graph_bytes = g.graph_bytes();
    st->workspace_bytes = sr.workspace_bytes;
    st->free_E = info.free_refs / 2u;
    st->terminal_edges = info.terminal_edges;
    st->rounds = sr.rounds;
    st->global_relabels = sr.relabels;
    st->map_bytes = N * 4u + (uint64_t)g.n * 4u;
    st->solve_seconds = sr.solve_s;
    st->final_relabel_seconds = sr.final_relabel_s;
    st->node_visits = sr.node_visits;
    st->pushes = sr.pushes;
    st->bfs_visits = sr.bfs_visits;
    st->bfs_levels = sr.bfs_levels;
    st->solve_device_ms = sr.solve_device_ms;
    st->discharge_ms = sr.discharge_ms;
    st->bfs_ms = sr.bfs_ms;
    st->discharge_launches = sr.discharge_launches;
    st->bfs_launches = sr.bfs_launches;
    st->engine = sr.engine;
    st->solve_blocks_per_sm = sr.blocks_per_sm;
    st->relabel_work_factor = sr.work_factor;
    st->chain_hops = sr.chain_hops;
    st->chain_max_active = sr.chain_max_active;
    st->sweep_ms = sr.sweep_ms;
    st->graphs_retired = sr.graphs_retired;
    st->bottom_up_steps = sr.bottom_up_steps;
    for (int k = 0; k < 3; ++k) {
        st->bfs_steps_by_frontier[k] = sr.step_cnt[k];
        st->bfs_ms_by_frontier[k] = sr.step_ms[k];
    }
    for (int k = 0; k < 3; ++k) {
        st->discharge_rounds_by_active[k] = sr.dround_cnt[k];
        st->discharge_ms_by_active[k] = sr.dround_ms[k];
    }
    st->bfs_tail_steps = sr.tail_steps;
    st->bfs_tail_levels = sr.tail_levels;
    st->relabel_tiles = sr.relabel_tiles;
    st->tile_steps = sr.tile_steps;
    st->tile_procs = sr.tile_procs;
    st->tile_loads = sr.tile_loads;
    st->tile_writes = sr.tile_writes;
    st->kernel_launches = launches;
    st->native_total_seconds = seconds_since(all0);
}

// Tuning of the persistent engine's free choices on one reduced graph (or a
// batch's segmented union): timed solves with the residuals and terminals
// restored before each, every candidate `reps` times, interleaved so slow
// drifts of the clock hit every candidate alike.  Stage 1: resident blocks per
// SM x relabel work factor with the base chaining; stage 2: chaining with the
// best pair.  Both stages also time `base` itself (the built-in rule), and the
// entry never replaces the rule by a setting that was not faster.  A
// candidate's zero fields take base's values.
struct TuneCand {
    int bps;
    double wf;
    int hops, cmax;
    std::vector<double> ms;
    SolveResult last;   // settings the solve actually used
};

double median_of(std::vector<double> v)
{
    std::sort(v.begin(), v.end());
    return v.size() % 2 ? v[v.size() / 2] : 0.5 * (v[v.size() / 2 - 1] + v[v.size() / 2]);
}

TuneEntry two_stage_tune(ReducedGraph& g, const Segments* segs, const gpupr_solve_options& base,
                         int32_t local_steps, int32_t reps, cudaStream_t s)
{
    DevBuf<uint32_t> res0(4u * (size_t)g.n, s);
    DevBuf<int32_t> term0(g.n, s);
    GPUPR_CUDA(cudaMemcpyAsync(res0.p, g.res.p, 16u * (size_t)g.n, cudaMemcpyDeviceToDevice, s));
    GPUPR_CUDA(cudaMemcpyAsync(term0.p, g.term.p, 4u * (size_t)g.n, cudaMemcpyDeviceToDevice, s));
    SolveWorkspace w;
    auto run = [&](std::vector<TuneCand>& cands) {
        for (int r = 0; r < reps; ++r)
            for (TuneCand& c : cands) {
                GPUPR_CUDA(cudaMemcpyAsync(g.res.p, res0.p, 16u * (size_t)g.n, cudaMemcpyDeviceToDevice, s));
                GPUPR_CUDA(cudaMemcpyAsync(g.term.p, term0.p, 4u * (size_t)g.n, cudaMemcpyDeviceToDevice, s));
                gpupr_solve_options o = base;
                o.local_steps = local_steps;
                o.engine = 2;
                if (c.bps) o.blocks_per_sm = c.bps;
                if (c.wf > 0) o.work_relabel_factor = c.wf;
                if (c.hops) o.chain_hops = c.hops;
                if (c.cmax) o.chain_max_active = c.cmax;
                SolveOptions opt = resolve_options(&o, local_steps, 1024, 2000000ull);
                SolveResult sr;
                solve_push_relabel(g.n, g.nbr.p, g.res.p, g.rev.p, g.pair.p, g.term.p, w, opt, s, sr, segs);
                c.ms.push_back(sr.solve_device_ms);
                c.last = sr;
            }
    };
    std::vector<TuneCand> c1;
    c1.push_back({0, 0.0, 0, 0, {}, {}});
    for (int bp : {1, 2, 3, 4})
        for (double f : {0.25, 0.5, 1.0, 2.0}) c1.push_back({bp, f, 0, 0, {}, {}});
    run(c1);
    size_t bi = 1;
    for (size_t i = 2; i < c1.size(); ++i)
        if (median_of(c1[i].ms) < median_of(c1[bi].ms)) bi = i;
    std::vector<TuneCand> c2;
    c2.push_back({0, 0.0, 0, 0, {}, {}});
    for (auto hc : {std::pair<int, int>{1, 1}, {4, 4096}, {4, 32768}, {8, 131072}})
        c2.push_back({c1[bi].bps, c1[bi].wf, hc.first, hc.second, {}, {}});
    run(c2);
    size_t bj = 0;
    for (size_t i = 1; i < c2.size(); ++i)
        if (median_of(c2[i].ms) < median_of(c2[bj].ms)) bj = i;
    const TuneCand& win = c2[bj];
    TuneEntry best;
    best.blocks_per_sm = win.last.blocks_per_sm;
    best.work_factor = win.last.work_factor;
    best.chain_hops = win.last.chain_hops;
    best.chain_max_active = win.last.chain_max_active;
    best.solve_ms = median_of(win.ms);
    std::vector<double> dflt = c1[0].ms;
    dflt.insert(dflt.end(), c2[0].ms.begin(), c2[0].ms.end());
    best.default_ms = median_of(dflt);
    return best;
}

// gpupr_autotune: one build, then the two-stage tuning of its solve; the
// entry is kept for the graph's size class.
TuneEntry run_autotune(const double* vertices, uint64_t nv, int v_dev, const int32_t* d_tets,
                       const int32_t* d_nbrs, uint64_t N, const uint8_t* labels, int l_dev,
                       double fill_T, int32_t local_steps, int32_t reps, cudaStream_t s)
{
    if (N == 0 || N > 0xFFFFFFFFull) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "autotune needs 1..2^32-1 tets"};
    if (!d_tets || !d_nbrs || !labels || (!vertices && nv))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL input"};
    if (!aligned(d_tets, 16) || !aligned(d_nbrs, 16))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be 16-byte aligned"};
    select_device_for(d_tets, "tets/neighbors");
    if (reps <= 0) reps = 3;
    if (reps > 50) reps = 50;
    DevBuf<uint8_t> dlab;
    DevBuf<double> dver;
    const uint8_t* d_labels = on_device(labels, N, l_dev, dlab, s);
    const double* d_vertices = on_device(vertices, nv * 3u, v_dev, dver, s);
    BuildInputs in{d_vertices, nv, d_tets, d_nbrs, d_labels, N, fill_T};
    ReducedGraph g;
    BuildInfo info;
    uint64_t launches = 0;
    build_reduced_graph(in, g, info, s, &launches);
    if (info.free_n == 0) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "autotune: the cut has no free tet"};
    // the built-in rule (an empty table: the rule, not an older entry)
    TuneEntry old;
    if (tune_lookup(g.n, &old)) {
        std::vector<TuneEntry> keep = tune_all();
        keep.erase(std::remove_if(keep.begin(), keep.end(),
                                  [&](const TuneEntry& e) { return e.size_class == size_class(g.n); }),
                   keep.end());
        tune_replace(keep);
    }
    gpupr_solve_options base{};
    TuneEntry best = two_stage_tune(g, nullptr, base, local_steps, reps, s);
    best.size_class = size_class(g.n);
    tune_store(best);
    return best;
}

// A batch packed, its union's reduced graph built, and each graph's range of
// reduced ids (the segments of the solve and of the per-graph flows).
struct PreparedBatch {
    DevBuf<uint8_t> dlab;
    DevBuf<double> dver;
    const uint8_t* d_labels = nullptr;
    DevBuf<unsigned long long> d_toff, d_voff, d_foff;
    DevBuf<uint32_t> d_soff;
    DevBuf<int32_t> gt, gn;
    ReducedGraph g;
    BuildInfo info;
    std::vector<unsigned long long> hc;   // free nodes per graph
    Segments segs;
};

// Checks the offsets and prepares the batch; stops after the build when no
// tet is free (pb.info.free_n == 0).
void prepare_batch(uint32_t G, const uint64_t* toff, const uint64_t* voff, const double* vertices,
                   int v_dev, const int32_t* d_tets_l, const int32_t* d_nbrs_l, const uint8_t* labels,
                   int l_dev, double fill_T, cudaStream_t s, PreparedBatch& pb, uint64_t* launches)
{
    if (toff[0] != 0 || voff[0] != 0) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "batch offsets must start at 0"};
    for (uint32_t k = 0; k < G; ++k)
        if (toff[k + 1] < toff[k] || voff[k + 1] < voff[k])
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "batch offsets must be non-decreasing"};
    const uint64_t N = toff[G], nv = voff[G];
    if (N > 0x7FFFFFFEull) throw Error{GPUPR_ERR_TOO_MANY_TETS, "batch exceeds 2^31-1 tets"};
    if (!d_tets_l || !d_nbrs_l || !labels || (!vertices && nv))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL batch array"};
    if (!aligned(d_tets_l, 16) || !aligned(d_nbrs_l, 16))
        throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be 16-byte aligned"};
    select_device_for(d_tets_l, "tets/neighbors");
    pb.d_labels = on_device(labels, N, l_dev, pb.dlab, s);
    const double* d_vertices = on_device(vertices, nv * 3u, v_dev, pb.dver, s);
    pb.d_toff = DevBuf<unsigned long long>(G + 1, s);
    pb.d_voff = DevBuf<unsigned long long>(G + 1, s);
    GPUPR_CUDA(cudaMemcpyAsync(pb.d_toff.p, toff, (G + 1) * 8u, cudaMemcpyHostToDevice, s));
    GPUPR_CUDA(cudaMemcpyAsync(pb.d_voff.p, voff, (G + 1) * 8u, cudaMemcpyHostToDevice, s));
    pb.gt = DevBuf<int32_t>(N * 4u, s);
    pb.gn = DevBuf<int32_t>(N * 4u, s);
    batch_pack(N, G, pb.d_toff.p, pb.d_voff.p, d_tets_l, d_nbrs_l, pb.gt.p, pb.gn.p, s, launches);
    BuildInputs in{d_vertices, nv, pb.gt.p, pb.gn.p, pb.d_labels, N, fill_T};
    in.want_base_node = true;
    build_reduced_graph(in, pb.g, pb.info, s, launches);
    if (pb.info.free_n == 0) return;
    // each graph's free nodes form one contiguous range of reduced ids
    DevBuf<unsigned long long> counts(G, s);
    batch_free_counts(G, pb.d_toff.p, pb.g.full_to_free.p, counts.p, s, launches);
    pb.hc.assign(G, 0);
    std::vector<unsigned long long> hfo(G + 1);
    std::vector<uint32_t> hso(G + 1);
    GPUPR_CUDA(cudaMemcpyAsync(pb.hc.data(), counts.p, G * 8u, cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaStreamSynchronize(s));
    hfo[0] = 0;
    for (uint32_t k = 0; k < G; ++k) hfo[k + 1] = hfo[k] + pb.hc[k];
    if (hfo[G] != pb.g.n) throw Error{GPUPR_ERR_INVARIANT, "batch free counts do not add up"};
    for (uint32_t k = 0; k <= G; ++k) hso[k] = (uint32_t)hfo[k];
    pb.d_foff = DevBuf<unsigned long long>(G + 1, s);
    pb.d_soff = DevBuf<uint32_t>(G + 1, s);
    GPUPR_CUDA(cudaMemcpyAsync(pb.d_foff.p, hfo.data(), (G + 1) * 8u, cudaMemcpyHostToDevice, s));
    GPUPR_CUDA(cudaMemcpyAsync(pb.d_soff.p, hso.data(), (G + 1) * 4u, cudaMemcpyHostToDevice, s));
    // the host vectors go out of scope: the copies must have read them
    GPUPR_CUDA(cudaStreamSynchronize(s));
    pb.segs.nseg = G;
    pb.segs.d_off = pb.d_soff.p;
}

// The options of a batch's solve: the caller's fields where set; else the
// batch tuning table's entry for the batch's size class (free nodes per
// graph); else, for a union of at least 16 graphs averaging under 1.5M tets,
// 8 chained hops in rounds of up to 131072 active nodes on 3 blocks per SM.
// That rule comes from B200 measurements with 64 graphs of 50k-4M tets
// (56.5M in all, mean 0.9M; median solve of 9 alternating runs): 73.3 ->
// 54.7 ms on one seeded batch, 86.3 -> 90.7 ms on another, against the
// union's own size rule; a single 5M-tet graph ran 3x slower with these
// settings, hence the mean-size bound.
gpupr_solve_options batch_options(const gpupr_solve_options* options, uint32_t G, uint64_t N,
                                  uint64_t free_n)
{
    gpupr_solve_options o{};
    if (options) o = *options;
    const bool caller_set = options && (options->chain_hops > 0 || options->chain_max_active > 0 ||
                                        options->blocks_per_sm > 0 || options->work_relabel_factor > 0);
    if (caller_set) return o;
    TuneEntry e;
    if (batch_tune_lookup(free_n / (G ? G : 1u), &e)) {
        o.blocks_per_sm = e.blocks_per_sm;
        o.work_relabel_factor = e.work_factor;
        o.chain_hops = e.chain_hops;
        o.chain_max_active = e.chain_max_active;
    } else if (G >= 16u && N / G < 1500000ull) {
        o.chain_hops = 8;
        o.chain_max_active = 131072;
        o.blocks_per_sm = 3;
    }
    return o;
}

}  // namespace

void run_graph_cut_batch(uint32_t G, const uint64_t* toff, const uint64_t* voff,
                         const double* vertices, int v_dev, const int32_t* d_tets_l,
                         const int32_t* d_nbrs_l, const uint8_t* labels, int l_dev, double fill_T,
                         const gpupr_solve_options* options, uint8_t* out, int out_dev,
                         cudaStream_t s, gpupr_batch_item* items, gpupr_cut_stats* st,
                         int max_blocks_per_sm)
{
    const auto all0 = std::chrono::steady_clock::now();
    if (!st || !items || !toff || !voff) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL batch argument"};
    std::memset(st, 0, sizeof(*st));
    std::memset(items, 0, sizeof(gpupr_batch_item) * G);
    if (!G) return;
    for (uint32_t k = 0; k < G; ++k) items[k].n_tets = toff[k + 1] >= toff[k] ? toff[k + 1] - toff[k] : 0;
    const uint64_t N = toff[G];
    st->n_full = N;
    st->threads = 1;
    st->local_steps = options && options->local_steps ? options->local_steps : 8;
    if (N == 0 && toff[0] == 0 && voff[0] == 0) return;
    if (!out) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL batch array"};
    uint64_t launches = 0;

    const auto b0 = std::chrono::steady_clock::now();
    Timer tb(s);
    PreparedBatch pb;
    prepare_batch(G, toff, voff, vertices, v_dev, d_tets_l, d_nbrs_l, labels, l_dev, fill_T, s, pb,
                  &launches);
    ReducedGraph& g = pb.g;
    const BuildInfo& info = pb.info;
    st->build_device_ms = tb.stop_ms();
    st->build_seconds = seconds_since(b0);
    st->full_E = info.full_refs / 2u;
    st->fixed_source = info.fixed_source;
    st->fixed_sink = info.fixed_sink;
    st->free_n = info.free_n;
    if (info.free_n == 0) {
        if (out_dev) GPUPR_CUDA(cudaMemcpyAsync(out, pb.d_labels, N, cudaMemcpyDeviceToDevice, s));
        else device_to_host(out, pb.d_labels, N, s);
        GPUPR_CUDA(cudaStreamSynchronize(s));
        st->kernel_launches = launches;
        st->native_total_seconds = seconds_since(all0);
        return;
    }
    const gpupr_solve_options bo = batch_options(options, G, N, info.free_n);
    SolveOptions opt = resolve_options(&bo, 8, 1024, 2000000ull);
    opt.max_blocks_per_sm = max_blocks_per_sm;
    SolveWorkspace w;
    SolveResult sr;
    solve_push_relabel(g.n, g.nbr.p, g.res.p, g.rev.p, g.pair.p, g.term.p, w, opt, s, sr, &pb.segs);
    launches += sr.launches;

    DevBuf<uint8_t> dout;
    uint8_t* d_out = out;
    if (!out_dev) {
        dout = DevBuf<uint8_t>(N, s);
        d_out = dout.p;
    }
    GPUPR_CUDA(cudaMemcpyAsync(d_out, pb.d_labels, N, cudaMemcpyDeviceToDevice, s));
    scatter_partition(g.n, g.free_old.p, w.height.p, d_out, s, &launches);

    // per-graph flows over each graph's contiguous free-node range
    DevBuf<unsigned long long> base(G, s);
    DevBuf<long long> raw(G, s);
    std::vector<unsigned long long> hb(G);
    std::vector<long long> hr(G);
    batch_flows(G, pb.d_foff.p, g.term.p, w.excess.p, g.base_node.p, raw.p, base.p, s, &launches);
    GPUPR_CUDA(cudaMemcpyAsync(hr.data(), raw.p, G * 8u, cudaMemcpyDeviceToHost, s));
    GPUPR_CUDA(cudaMemcpyAsync(hb.data(), base.p, G * 8u, cudaMemcpyDeviceToHost, s));
    if (!out_dev) device_to_host(out, d_out, N, s);
    GPUPR_CUDA(cudaStreamSynchronize(s));
    for (uint32_t k = 0; k < G; ++k) {
        items[k].raw_flow = hr[k];
        items[k].adjusted_flow = hr[k] + (long long)hb[k];
        items[k].free_n = pb.hc[k];
    }
    st->raw_flow = sr.raw_flow;
    st->adjusted_flow = sr.raw_flow + info.terminal_base_flow;
    st->graph_bytes = g.graph_bytes();
    st->workspace_bytes = sr.workspace_bytes;
    st->free_E = info.free_refs / 2u;
    st->terminal_edges = info.terminal_edges;
    st->rounds = sr.rounds;
    st->global_relabels = sr.relabels;
    st->map_bytes = N * 4u + (uint64_t)g.n * 4u;
    st->solve_seconds = sr.solve_s;
    st->node_visits = sr.node_visits;
    st->pushes = sr.pushes;
    st->bfs_visits = sr.bfs_visits;
    st->bfs_levels = sr.bfs_levels;
    st->solve_device_ms = sr.solve_device_ms;
    st->discharge_ms = sr.discharge_ms;
    st->bfs_ms = sr.bfs_ms;
    st->engine = sr.engine;
    st->solve_blocks_per_sm = sr.blocks_per_sm;
    st->relabel_work_factor = sr.work_factor;
    st->chain_hops = sr.chain_hops;
    st->chain_max_active = sr.chain_max_active;
    st->sweep_ms = sr.sweep_ms;
    st->graphs_retired = sr.graphs_retired;
    st->bottom_up_steps = sr.bottom_up_steps;
    for (int k = 0; k < 3; ++k) {
        st->bfs_steps_by_frontier[k] = sr.step_cnt[k];
        st->bfs_ms_by_frontier[k] = sr.step_ms[k];
    }
    for (int k = 0; k < 3; ++k) {
        st->discharge_rounds_by_active[k] = sr.dround_cnt[k];
        st->discharge_ms_by_active[k] = sr.dround_ms[k];
    }
    st->bfs_tail_steps = sr.tail_steps;
    st->bfs_tail_levels = sr.tail_levels;
    st->relabel_tiles = sr.relabel_tiles;
    st->tile_steps = sr.tile_steps;
    st->tile_procs = sr.tile_procs;
    st->tile_loads = sr.tile_loads;
    st->tile_writes = sr.tile_writes;
    st->kernel_launches = launches;
    st->native_total_seconds = seconds_since(all0);
}

// gpupr_autotune_batch: one pack and build, then the two-stage tuning of the
// segmented solve against the batch rule; the entry is kept for the batch's
// size class (free nodes per graph).
TuneEntry run_autotune_batch(uint32_t G, const uint64_t* toff, const uint64_t* voff,
                             const double* vertices, int v_dev, const int32_t* d_tets_l,
                             const int32_t* d_nbrs_l, const uint8_t* labels, int l_dev, double fill_T,
                             int32_t local_steps, int32_t reps, cudaStream_t s)
{
    if (!G || !toff || !voff) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL batch argument"};
    if (reps <= 0) reps = 3;
    if (reps > 50) reps = 50;
    uint64_t launches = 0;
    PreparedBatch pb;
    prepare_batch(G, toff, voff, vertices, v_dev, d_tets_l, d_nbrs_l, labels, l_dev, fill_T, s, pb,
                  &launches);
    if (pb.info.free_n == 0) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "autotune: the batch has no free tet"};
    const uint64_t mean_free = pb.info.free_n / G;
    // the rule, not an older entry of this class
    std::vector<TuneEntry> keep = batch_tune_all();
    keep.erase(std::remove_if(keep.begin(), keep.end(),
                              [&](const TuneEntry& e) { return e.size_class == size_class((uint32_t)mean_free); }),
               keep.end());
    batch_tune_replace(keep);
    const gpupr_solve_options base = batch_options(nullptr, G, toff[G], pb.info.free_n);
    TuneEntry best = two_stage_tune(pb.g, &pb.segs, base, local_steps, reps, s);
    best.size_class = size_class((uint32_t)mean_free);
    batch_tune_store(best);
    return best;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

void* pool_alloc(size_t bytes, cudaStream_t s)
{
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, device_pool(), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{GPUPR_ERR_OUT_OF_MEMORY, "insufficient VRAM for reduced graph + solver (" +
                                                 std::to_string(bytes) + " bytes: " +
                                                 cudaGetErrorString(e) + ")"};
    }
    return p;
}

void pool_free(void* p, cudaStream_t s)
{
    if (p) cudaFreeAsync(p, s);
}

}  // namespace gpupr

using namespace gpupr;

extern "C" {

const char* gpupr_status_string(gpupr_status status)
{
    switch (status) {
    case GPUPR_OK: return "ok";
    case GPUPR_ERR_INVALID_ARGUMENT: return "invalid argument";
    case GPUPR_ERR_NEIGHBOR_RANGE: return "neighbor out of range";
    case GPUPR_ERR_REFS_ODD: return "neighbor reference count not even";
    case GPUPR_ERR_BUILD: return "invalid graph reduction/capacity state";
    case GPUPR_ERR_FREE_REFS_ODD: return "free reference count not even";
    case GPUPR_ERR_TOO_MANY_NODES: return ">INT32_MAX reduced nodes unsupported";
    case GPUPR_ERR_NO_REVERSE: return "device invariant failed (asymmetric adjacency)";
    case GPUPR_ERR_OUT_OF_MEMORY: return "insufficient VRAM for reduced graph + solver";
    case GPUPR_ERR_MAX_ROUNDS: return "GPUPr-FAST-v6.30 max macro rounds exceeded";
    case GPUPR_ERR_INVARIANT: return "device invariant failed";
    case GPUPR_ERR_CUDA: return "CUDA failure";
    case GPUPR_ERR_TIMEOUT: return "time limit exceeded";
    case GPUPR_ERR_TOO_MANY_TETS: return ">2^32 full tets unsupported";
    }
    return "unknown status";
}

const char* gpupr_last_error(void) { return g_last_error.c_str(); }

int gpupr_abi_version(void) { return GPUPR_ABI_VERSION; }

gpupr_status gpupr_graph_cut(const double* vertices, uint64_t n_vertices, int vertices_on_device,
                             const int32_t* d_tets, const int32_t* d_neighbors, uint64_t n_tets,
                             const uint8_t* labels, int labels_on_device, double fill_T,
                             int32_t threads, int32_t global_relabel_period, uint64_t max_rounds,
                             int32_t local_steps, uint8_t* out_labels, int out_on_device,
                             void* stream, gpupr_cut_stats* stats)
{
    return guarded([&] {
        run_graph_cut(vertices, n_vertices, vertices_on_device, d_tets, d_neighbors, n_tets, labels,
                      labels_on_device, fill_T, threads, global_relabel_period, max_rounds,
                      local_steps, nullptr, out_labels, out_on_device,
                      static_cast<cudaStream_t>(stream), stats);
    });
}

gpupr_status gpupr_graph_cut_ex(const double* vertices, uint64_t n_vertices, int vertices_on_device,
                                const int32_t* d_tets, const int32_t* d_neighbors, uint64_t n_tets,
                                const uint8_t* labels, int labels_on_device, double fill_T,
                                int32_t threads, const gpupr_solve_options* options,
                                uint8_t* out_labels, int out_on_device, void* stream,
                                gpupr_cut_stats* stats)
{
    return guarded([&] {
        const int32_t ls = options && options->local_steps ? options->local_steps : 8;
        const int32_t per = options && options->global_relabel_period ? options->global_relabel_period : 1024;
        const uint64_t mr = options && options->max_rounds ? options->max_rounds : 2000000ull;
        run_graph_cut(vertices, n_vertices, vertices_on_device, d_tets, d_neighbors, n_tets, labels,
                      labels_on_device, fill_T, threads, per, mr, ls, options, out_labels,
                      out_on_device, static_cast<cudaStream_t>(stream), stats);
    });
}

gpupr_status gpupr_graph_cut_batch(uint32_t n_graphs, const uint64_t* tet_offsets,
                                   const uint64_t* vertex_offsets, const double* vertices,
                                   int vertices_on_device, const int32_t* d_tets,
                                   const int32_t* d_neighbors, const uint8_t* labels,
                                   int labels_on_device, double fill_T,
                                   const gpupr_solve_options* options, uint8_t* out_labels,
                                   int out_on_device, void* stream, gpupr_batch_item* items,
                                   gpupr_cut_stats* stats)
{
    return guarded([&] {
        run_graph_cut_batch(n_graphs, tet_offsets, vertex_offsets, vertices, vertices_on_device,
                            d_tets, d_neighbors, labels, labels_on_device, fill_T, options,
                            out_labels, out_on_device, static_cast<cudaStream_t>(stream), items,
                            stats);
    });
}

gpupr_status gpupr_build_reduced(const double* vertices, uint64_t n_vertices, int vertices_on_device,
                                 const int32_t* d_tets, const int32_t* d_neighbors, uint64_t n_tets,
                                 const uint8_t* labels, int labels_on_device, double fill_T,
                                 int32_t* full_to_free, uint32_t* free_old, int32_t* nbr,
                                 uint32_t* res, int32_t* term, uint8_t* rev, int64_t* info_out,
                                 void* stream)
{
    return guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (!info_out) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "info pointer is NULL"};
        std::memset(info_out, 0, 8 * sizeof(int64_t));
        info_out[7] = (int64_t)n_tets;
        if (n_tets == 0) return;
        if (n_tets > 0xFFFFFFFFull) throw Error{GPUPR_ERR_TOO_MANY_TETS, ">2^32 full tets unsupported"};
        if (!d_tets || !d_neighbors || !labels || (!vertices && n_vertices))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL input"};
        if (!aligned(d_tets, 16) || !aligned(d_neighbors, 16))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be 16-byte aligned"};
        select_device_for(d_tets, "tets/neighbors");
        DevBuf<uint8_t> dlab;
        DevBuf<double> dver;
        const uint8_t* d_labels = on_device(labels, n_tets, labels_on_device, dlab, s);
        const double* d_vertices = on_device(vertices, n_vertices * 3u, vertices_on_device, dver, s);
        BuildInputs in{d_vertices, n_vertices, d_tets, d_neighbors, d_labels, n_tets, fill_T};
        ReducedGraph g;
        BuildInfo info;
        uint64_t launches = 0;
        build_reduced_graph(in, g, info, s, &launches);
        info_out[0] = (int64_t)info.free_n;
        info_out[1] = (int64_t)info.fixed_source;
        info_out[2] = (int64_t)info.fixed_sink;
        info_out[3] = (int64_t)info.full_refs;
        info_out[4] = (int64_t)info.free_refs;
        info_out[5] = (int64_t)info.terminal_edges;
        info_out[6] = info.terminal_base_flow;
        const size_t F = info.free_n;
        if (full_to_free)
            GPUPR_CUDA(cudaMemcpyAsync(full_to_free, g.full_to_free.p, n_tets * 4u, cudaMemcpyDeviceToHost, s));
        if (F) {
            if (free_old) GPUPR_CUDA(cudaMemcpyAsync(free_old, g.free_old.p, F * 4u, cudaMemcpyDeviceToHost, s));
            if (nbr) GPUPR_CUDA(cudaMemcpyAsync(nbr, g.nbr.p, F * 16u, cudaMemcpyDeviceToHost, s));
            if (res) GPUPR_CUDA(cudaMemcpyAsync(res, g.res.p, F * 16u, cudaMemcpyDeviceToHost, s));
            if (term) GPUPR_CUDA(cudaMemcpyAsync(term, g.term.p, F * 4u, cudaMemcpyDeviceToHost, s));
            if (rev) GPUPR_CUDA(cudaMemcpyAsync(rev, g.rev.p, F, cudaMemcpyDeviceToHost, s));
        }
        GPUPR_CUDA(cudaStreamSynchronize(s));
    });
}

gpupr_status gpupr_solve_reduced(uint32_t n, int32_t* d_neighbors, uint32_t* d_residual,
                                 int32_t* d_terminal, uint8_t* h_partition,
                                 int32_t global_relabel_period, uint64_t max_rounds,
                                 int32_t local_steps, int64_t* d_excess_out, void* stream,
                                 gpupr_cut_stats* stats)
{
    return guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        if (!n) return;
        if (!d_neighbors || !d_residual || !d_terminal || !h_partition)
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "GPUPr-FAST-v6.30 null graph pointer"};
        if (!aligned(d_neighbors, 16) || !aligned(d_residual, 16))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "graph rows must be 16-byte aligned"};
        if (n > 0x7FFFFFFFu) throw Error{GPUPR_ERR_TOO_MANY_NODES, ">INT32_MAX reduced nodes unsupported"};
        select_device_for(d_neighbors, "graph");
        uint64_t launches = 0;
        DevBuf<uint8_t> rev(n, s);
        DevBuf<uint32_t> pair((size_t)n * 4u, s);
        compute_reverse_slots(n, reinterpret_cast<const int4*>(d_neighbors), d_residual, rev.p,
                              pair.p, s, &launches);
        const SolveOptions opt = resolve_options(nullptr, local_steps, global_relabel_period, max_rounds);
        SolveWorkspace w;
        SolveResult sr;
        solve_push_relabel(n, reinterpret_cast<const int4*>(d_neighbors), d_residual, rev.p,
                           pair.p, d_terminal, w, opt, s, sr);
        launches += sr.launches;
        DevBuf<uint8_t> part(n, s);
        partition_from_height(n, w.height.p, part.p, s, &launches);
        GPUPR_CUDA(cudaMemcpyAsync(h_partition, part.p, n, cudaMemcpyDeviceToHost, s));
        if (d_excess_out)
            GPUPR_CUDA(cudaMemcpyAsync(d_excess_out, w.excess.p, (size_t)n * 8u, cudaMemcpyDeviceToDevice, s));
        GPUPR_CUDA(cudaStreamSynchronize(s));
        if (stats) {
            stats->raw_flow = sr.raw_flow;
            stats->adjusted_flow = sr.raw_flow;
            stats->workspace_bytes = sr.workspace_bytes;
            stats->rounds = sr.rounds;
            stats->global_relabels = sr.relabels;
            stats->local_steps = local_steps;
            stats->solve_seconds = sr.solve_s;
            stats->final_relabel_seconds = sr.final_relabel_s;
            stats->free_n = n;
            stats->node_visits = sr.node_visits;
            stats->pushes = sr.pushes;
            stats->bfs_visits = sr.bfs_visits;
            stats->bfs_levels = sr.bfs_levels;
            stats->solve_device_ms = sr.solve_device_ms;
            stats->discharge_ms = sr.discharge_ms;
            stats->bfs_ms = sr.bfs_ms;
            stats->discharge_launches = sr.discharge_launches;
            stats->bfs_launches = sr.bfs_launches;
            stats->engine = sr.engine;
            stats->solve_blocks_per_sm = sr.blocks_per_sm;
            stats->relabel_work_factor = sr.work_factor;
            stats->chain_hops = sr.chain_hops;
            stats->chain_max_active = sr.chain_max_active;
            stats->sweep_ms = sr.sweep_ms;
            stats->graphs_retired = sr.graphs_retired;
            stats->bottom_up_steps = sr.bottom_up_steps;
            for (int k = 0; k < 3; ++k) {
                stats->bfs_steps_by_frontier[k] = sr.step_cnt[k];
                stats->bfs_ms_by_frontier[k] = sr.step_ms[k];
            }
            for (int k = 0; k < 3; ++k) {
                stats->discharge_rounds_by_active[k] = sr.dround_cnt[k];
                stats->discharge_ms_by_active[k] = sr.dround_ms[k];
            }
            stats->bfs_tail_steps = sr.tail_steps;
            stats->bfs_tail_levels = sr.tail_levels;
            stats->relabel_tiles = sr.relabel_tiles;
            stats->tile_steps = sr.tile_steps;
            stats->tile_procs = sr.tile_procs;
            stats->tile_loads = sr.tile_loads;
            stats->tile_writes = sr.tile_writes;
            stats->kernel_launches = launches;
        }
    });
}

gpupr_status gpupr_solve_ell(uint32_t n, const int32_t* d_nbr, const uint32_t* d_cap,
                             const uint32_t* d_src, const uint32_t* d_snk,
                             const gpupr_solve_options* options, int64_t* max_flow,
                             uint8_t* d_partition, void* stream, gpupr_cut_stats* stats)
{
    return guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        if (max_flow) *max_flow = 0;
        if (!n) return;
        if (!d_nbr || !d_cap || !d_src || !d_snk || !max_flow || !d_partition)
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL graph pointer"};
        if (!aligned(d_nbr, 16) || !aligned(d_cap, 16))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "graph rows must be 16-byte aligned"};
        if (n > 0x7FFFFFFFu) throw Error{GPUPR_ERR_TOO_MANY_NODES, ">INT32_MAX nodes unsupported"};
        select_device_for(d_nbr, "graph");
        uint64_t launches = 0;
        DevBuf<uint32_t> res((size_t)n * 4u, s);
        DevBuf<int32_t> term(n, s);
        DevBuf<uint8_t> rev(n, s);
        DevBuf<uint32_t> pair((size_t)n * 4u, s);
        const int64_t base = prepare_raw_graph(n, d_cap, d_src, d_snk, d_nbr, res.p, term.p, s, &launches);
        compute_reverse_slots(n, reinterpret_cast<const int4*>(d_nbr), res.p, rev.p, pair.p, s, &launches);
        const SolveOptions opt = resolve_options(options, 8, 1024, 2000000ull);
        SolveWorkspace w;
        SolveResult sr;
        solve_push_relabel(n, reinterpret_cast<const int4*>(d_nbr), res.p, rev.p, pair.p, term.p, w,
                           opt, s, sr);
        launches += sr.launches;
        partition_from_height(n, w.height.p, d_partition, s, &launches);
        GPUPR_CUDA(cudaStreamSynchronize(s));
        *max_flow = base + sr.raw_flow;
        if (stats) {
            stats->adjusted_flow = base + sr.raw_flow;
            stats->raw_flow = sr.raw_flow;
            stats->graph_bytes = res.bytes() + term.bytes() + rev.bytes() + pair.bytes();
            stats->workspace_bytes = sr.workspace_bytes;
            stats->rounds = sr.rounds;
            stats->global_relabels = sr.relabels;
            stats->local_steps = opt.local_steps;
            stats->solve_seconds = sr.solve_s;
            stats->final_relabel_seconds = sr.final_relabel_s;
            stats->free_n = n;
            stats->node_visits = sr.node_visits;
            stats->pushes = sr.pushes;
            stats->bfs_visits = sr.bfs_visits;
            stats->bfs_levels = sr.bfs_levels;
            stats->solve_device_ms = sr.solve_device_ms;
            stats->discharge_ms = sr.discharge_ms;
            stats->bfs_ms = sr.bfs_ms;
            stats->discharge_launches = sr.discharge_launches;
            stats->bfs_launches = sr.bfs_launches;
            stats->engine = sr.engine;
            stats->solve_blocks_per_sm = sr.blocks_per_sm;
            stats->relabel_work_factor = sr.work_factor;
            stats->chain_hops = sr.chain_hops;
            stats->chain_max_active = sr.chain_max_active;
            stats->sweep_ms = sr.sweep_ms;
            stats->graphs_retired = sr.graphs_retired;
            stats->bottom_up_steps = sr.bottom_up_steps;
            for (int k = 0; k < 3; ++k) {
                stats->bfs_steps_by_frontier[k] = sr.step_cnt[k];
                stats->bfs_ms_by_frontier[k] = sr.step_ms[k];
            }
            for (int k = 0; k < 3; ++k) {
                stats->discharge_rounds_by_active[k] = sr.dround_cnt[k];
                stats->discharge_ms_by_active[k] = sr.dround_ms[k];
            }
            stats->bfs_tail_steps = sr.tail_steps;
            stats->bfs_tail_levels = sr.tail_levels;
            stats->relabel_tiles = sr.relabel_tiles;
            stats->tile_steps = sr.tile_steps;
            stats->tile_procs = sr.tile_procs;
            stats->tile_loads = sr.tile_loads;
            stats->tile_writes = sr.tile_writes;
            stats->kernel_launches = launches;
        }
    });
}

gpupr_status gpupr_surface_count(const uint8_t* labels, int labels_on_device, const double* vertices,
                                 uint64_t n_vertices, int vertices_on_device, const int32_t* d_tets,
                                 const int32_t* d_neighbors, uint64_t n_tets, uint64_t* n_faces,
                                 uint64_t* n_used, void* stream)
{
    return guarded([&] {
        if (!n_faces || !n_used) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL count pointer"};
        *n_faces = 0;
        *n_used = 0;
        if (n_tets && (!d_tets || !d_neighbors || !labels))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be contiguous CUDA int32 Nx4 with same N"};
        if (n_tets) {
            if (!aligned(d_tets, 16) || !aligned(d_neighbors, 16))
                throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets/neighbors must be 16-byte aligned"};
            select_device_for(d_tets, "tets/neighbors");
        }
        surface_count(labels, labels_on_device, vertices, n_vertices, vertices_on_device, d_tets,
                      d_neighbors, n_tets, n_faces, n_used, static_cast<cudaStream_t>(stream));
    });
}

gpupr_status gpupr_surface_fetch(int32_t* faces, double* vertices_out, int out_on_device, void* stream)
{
    return guarded([&] { surface_fetch(faces, vertices_out, out_on_device, static_cast<cudaStream_t>(stream)); });
}

gpupr_status gpupr_solve_reduced_noalloc(uint32_t n, int32_t* d_neighbors, uint32_t* d_residual,
                                         int32_t* d_terminal, uint8_t* d_partition,
                                         int32_t global_relabel_period, uint64_t max_rounds,
                                         int32_t local_steps, void* stream, gpupr_cut_stats* stats)
{
    return guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        if (!n) return;
        if (!d_neighbors || !d_residual || !d_terminal || !d_partition)
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "GPUPr-FAST-v6.30 null graph pointer"};
        if (!aligned(d_neighbors, 16) || !aligned(d_residual, 16))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "graph rows must be 16-byte aligned"};
        select_device_for(d_neighbors, "graph");
        const SolveOptions opt = resolve_options(nullptr, local_steps, global_relabel_period, max_rounds);
        SolveResult sr;
        solve_reduced_noalloc(n, d_neighbors, d_residual, d_terminal, d_partition, opt, s, sr);
        if (stats) {
            stats->raw_flow = sr.raw_flow;
            stats->adjusted_flow = sr.raw_flow;
            stats->rounds = sr.rounds;
            stats->global_relabels = sr.relabels;
            stats->local_steps = local_steps;
            stats->solve_seconds = sr.solve_s;
            stats->free_n = n;
            stats->node_visits = sr.node_visits;
            stats->pushes = sr.pushes;
            stats->bfs_visits = sr.bfs_visits;
            stats->bfs_levels = sr.bfs_levels;
            stats->kernel_launches = sr.launches;
        }
    });
}

gpupr_status gpupr_noalloc_prepare(uint64_t* scratch_bytes)
{
    return guarded([&] {
        const uint64_t b = noalloc_prepare();
        if (scratch_bytes) *scratch_bytes = b;
    });
}

gpupr_status gpupr_upload_topology(const void* host, uint64_t rows, int64_t row_stride_bytes,
                                   int64_t col_stride_bytes, int32_t elem_bytes, int32_t* d_out,
                                   void* stream)
{
    return guarded([&] {
        if (!rows) return;
        if (!host || !d_out) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL topology pointer"};
        if (elem_bytes != 4 && elem_bytes != 8)
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "topology elements must be int32 or int64"};
        if (!aligned(d_out, 16)) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "d_out must be 16-byte aligned"};
        select_device_for(d_out, "d_out");
        upload_topology(d_out, host, rows, row_stride_bytes, col_stride_bytes, elem_bytes,
                        static_cast<cudaStream_t>(stream));
    });
}

gpupr_status gpupr_edge_audit(const int32_t* faces, uint64_t n_faces, int faces_on_device,
                              uint64_t* bad_groups, uint64_t* table_bytes, void* stream)
{
    return guarded([&] {
        if (!bad_groups || !table_bytes) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL result pointer"};
        *bad_groups = 0;
        *table_bytes = 0;
        if (!n_faces) return;
        if (!faces) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "faces pointer is NULL"};
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (faces_on_device) select_device_for(faces, "faces");
        DevBuf<int32_t> dfaces;
        const int32_t* d = on_device(faces, n_faces * 3u, faces_on_device, dfaces, s);
        edge_audit(d, n_faces, s, bad_groups, table_bytes, nullptr);
    });
}

gpupr_status gpupr_sample_tet_labels(const gpupr_brick_grid* grid, const double* vertices,
                                     uint64_t n_vertices, int vertices_on_device,
                                     const int32_t* tets, uint64_t n_tets, int tets_on_device,
                                     const double* bbox_min, const double* bbox_max,
                                     double padding, double threshold, uint8_t* labels_out,
                                     int labels_on_device, float* udf_out, void* stream)
{
    return guarded([&] {
        if (!grid) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "SparseUDF.sample_tet_labels: grid is empty"};
        if (!bbox_min || !bbox_max) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "SparseUDF.sample_tet_labels: bbox must have length 3"};
        if (!(grid->voxel_size > 0.0) || grid->dims[0] < 0 || grid->dims[1] < 0 || grid->dims[2] < 0)
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "invalid brick grid"};
        const uint64_t cells = (uint64_t)grid->dims[0] * (uint64_t)grid->dims[1] * (uint64_t)grid->dims[2];
        if (cells && !grid->table) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "invalid brick grid"};
        if (grid->n_bricks && !grid->values) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "invalid brick grid"};
        if (n_tets && (!tets || !labels_out || (!vertices && n_vertices)))
            throw Error{GPUPR_ERR_INVALID_ARGUMENT, "NULL input"};
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (tets_on_device && n_tets) {
            if (!aligned(tets, 16)) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "tets must be 16-byte aligned"};
            select_device_for(tets, "tets");
        } else if (grid->on_device && cells) {
            select_device_for(grid->table, "grid");
        }
        DevBuf<int32_t> dtab, dtets;
        DevBuf<float> dval, dudf;
        DevBuf<double> dver;
        DevBuf<uint8_t> dlab;
        BrickGridDesc g{};
        g.voxel_size = grid->voxel_size;
        for (int k = 0; k < 3; ++k) {
            g.origin[k] = grid->origin[k];
            g.dims[k] = grid->dims[k];
        }
        g.background = grid->background;
        // the grid is checked before the tets are touched, like the reference
        g.d_table = on_device(grid->table, cells, grid->on_device, dtab, s);
        g.d_values = on_device(grid->values, grid->n_bricks * 512u, grid->on_device, dval, s);
        const double* d_v = on_device(vertices, n_vertices * 3u, vertices_on_device, dver, s);
        const int32_t* d_t = on_device(tets, n_tets * 4u, tets_on_device, dtets, s);
        uint8_t* d_l = labels_out;
        float* d_u = udf_out;
        if (!labels_on_device && n_tets) {
            dlab = DevBuf<uint8_t>(n_tets, s);
            d_l = dlab.p;
            if (udf_out) {
                dudf = DevBuf<float>(n_tets, s);
                d_u = dudf.p;
            }
        }
        sample_tet_labels(g, d_v, n_vertices, d_t, n_tets, bbox_min, bbox_max, padding, threshold, d_l,
                          d_u, s, nullptr);
        if (!labels_on_device && n_tets) {
            device_to_host(labels_out, d_l, n_tets, s);
            if (udf_out) device_to_host(udf_out, d_u, n_tets * 4u, s);
        }
        GPUPR_CUDA(cudaStreamSynchronize(s));
    });
}

gpupr_status gpupr_autotune(const double* vertices, uint64_t n_vertices, int vertices_on_device,
                            const int32_t* d_tets, const int32_t* d_neighbors, uint64_t n_tets,
                            const uint8_t* labels, int labels_on_device, double fill_T,
                            int32_t local_steps, int32_t reps, gpupr_tune_entry* chosen,
                            void* stream)
{
    return guarded([&] {
        const TuneEntry e = run_autotune(vertices, n_vertices, vertices_on_device, d_tets, d_neighbors,
                                         n_tets, labels, labels_on_device, fill_T,
                                         local_steps > 0 ? local_steps : 8, reps,
                                         static_cast<cudaStream_t>(stream));
        if (chosen) {
            chosen->size_class = e.size_class;
            chosen->blocks_per_sm = e.blocks_per_sm;
            chosen->work_relabel_factor = e.work_factor;
            chosen->solve_ms = e.solve_ms;
            chosen->default_ms = e.default_ms;
            chosen->chain_hops = e.chain_hops;
            chosen->chain_max_active = e.chain_max_active;
        }
    });
}

namespace {
void export_entries(const std::vector<gpupr::TuneEntry>& all, gpupr_tune_entry* entries,
                    uint32_t capacity, uint32_t* count)
{
    *count = (uint32_t)all.size();
    for (uint32_t i = 0; i < all.size() && i < capacity && entries; ++i) {
        entries[i].size_class = all[i].size_class;
        entries[i].blocks_per_sm = all[i].blocks_per_sm;
        entries[i].work_relabel_factor = all[i].work_factor;
        entries[i].solve_ms = all[i].solve_ms;
        entries[i].default_ms = all[i].default_ms;
        entries[i].chain_hops = all[i].chain_hops;
        entries[i].chain_max_active = all[i].chain_max_active;
    }
}

std::vector<gpupr::TuneEntry> import_entries(const gpupr_tune_entry* entries, uint32_t count)
{
    if (count && !entries) throw gpupr::Error{GPUPR_ERR_INVALID_ARGUMENT, "entries pointer is NULL"};
    std::vector<gpupr::TuneEntry> v(count);
    for (uint32_t i = 0; i < count; ++i) {
        v[i].size_class = entries[i].size_class;
        v[i].blocks_per_sm = entries[i].blocks_per_sm;
        v[i].work_factor = entries[i].work_relabel_factor;
        v[i].solve_ms = entries[i].solve_ms;
        v[i].default_ms = entries[i].default_ms;
        v[i].chain_hops = entries[i].chain_hops;
        v[i].chain_max_active = entries[i].chain_max_active;
    }
    return v;
}
}  // namespace

gpupr_status gpupr_tune_table(gpupr_tune_entry* entries, uint32_t capacity, uint32_t* count)
{
    return guarded([&] {
        if (!count) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "count pointer is NULL"};
        export_entries(tune_all(), entries, capacity, count);
    });
}

gpupr_status gpupr_tune_table_set(const gpupr_tune_entry* entries, uint32_t count)
{
    return guarded([&] { tune_replace(import_entries(entries, count)); });
}

gpupr_status gpupr_autotune_batch(uint32_t n_graphs, const uint64_t* tet_offsets,
                                  const uint64_t* vertex_offsets, const double* vertices,
                                  int vertices_on_device, const int32_t* d_tets,
                                  const int32_t* d_neighbors, const uint8_t* labels,
                                  int labels_on_device, double fill_T, int32_t local_steps,
                                  int32_t reps, gpupr_tune_entry* chosen, void* stream)
{
    return guarded([&] {
        const TuneEntry e = run_autotune_batch(n_graphs, tet_offsets, vertex_offsets, vertices,
                                               vertices_on_device, d_tets, d_neighbors, labels,
                                               labels_on_device, fill_T, local_steps > 0 ? local_steps : 8,
                                               reps, static_cast<cudaStream_t>(stream));
        if (chosen) {
            uint32_t one = 0;
            export_entries({e}, chosen, 1, &one);
        }
    });
}

gpupr_status gpupr_batch_tune_table(gpupr_tune_entry* entries, uint32_t capacity, uint32_t* count)
{
    return guarded([&] {
        if (!count) throw Error{GPUPR_ERR_INVALID_ARGUMENT, "count pointer is NULL"};
        export_entries(batch_tune_all(), entries, capacity, count);
    });
}

gpupr_status gpupr_batch_tune_table_set(const gpupr_tune_entry* entries, uint32_t count)
{
    return guarded([&] { batch_tune_replace(import_entries(entries, count)); });
}

gpupr_status gpupr_release_cached_memory(void)
{
    return guarded([&] {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        for (int d = 0; d < 64; ++d)
            if (g_pools[d]) GPUPR_CUDA(cudaMemPoolTrimTo(g_pools[d], 0));
    });
}

gpupr_status gpupr_selftest_bounded_wait(uint32_t limit_us, void* stream)
{
    gpupr_status result = GPUPR_OK;
    gpupr_status st = guarded([&] {
        result = bounded_wait_selftest(limit_us, static_cast<cudaStream_t>(stream));
        if (result == GPUPR_ERR_TIMEOUT) g_last_error = "bounded wait gave up after the limit";
    });
    if (st != GPUPR_OK) return st;
    if (result == GPUPR_ERR_TIMEOUT) g_last_error = "bounded wait gave up after the limit";
    return result;
}

}  // extern "C"
