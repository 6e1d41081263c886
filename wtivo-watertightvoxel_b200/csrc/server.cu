// server.cu -- continuous-batching serving loop for graph cuts.
//
// Clients submit cut requests (one cell graph each, host arrays) at any time;
// the server borrows the arrays (no host copy) until the request is done and
// writes the labels straight into the caller's output array.
//
// Requests go to one of two lanes by size (tets below the split: the small
// lane; the rest: the large lane; split 0 = one lane).  Each lane has two
// threads and two streams:
//
//   stager  admits the lane's pending requests in arrival order while their
//           estimated device footprint fits the HBM budget left by every
//           batch staged or being solved on either lane (one batch shares
//           fill_T), copies each request's arrays into the lane's packed
//           device batch on its upload stream, and hands the batch over (one
//           staged batch per lane at most);
//   solver  cuts the staged batch as one segmented graph (run_graph_cut_batch:
//           one build, one persistent solve that retires each graph once it is
//           finished, per-graph flows), copies each request's labels out and
//           publishes the results.
//
// So uploads overlap solves, requests that arrive while a batch runs join the
// next one, and a small request never waits for a large one's solve: the two
// lanes' solves run at the same time.  A small request that arrives while the
// small lane has work in flight and the large lane has none takes the large
// lane (three times the small lane's grid), so a backlog of small requests
// does not pile up on one resident block per SM while most of the GPU idles.  Their persistent grids are capped so
// that both fit on the GPU together (small lane 1 resident block per SM, large
// lane the kernel's occupancy limit minus one): every block of both grids can
// be resident at once, whichever launches first, so neither grid's barrier
// waits on blocks that cannot be scheduled.  Results are exact: the cut of a
// graph does not depend on what else is in its batch or on the other lane.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gpupr_internal.cuh"
#include "wtivo_gpupr.h"

struct gpupr_server {
    using Clock = std::chrono::steady_clock;
    struct Request {
        uint64_t id = 0;
        const double* V = nullptr;
        const int32_t* T = nullptr;
        const int32_t* Nb = nullptr;
        const uint8_t* L = nullptr;
        uint8_t* out = nullptr;
        uint64_t nv = 0, n = 0;
        double fill_T = 10.0;
        int lane = 0;
        Clock::time_point t_submit, t_start;
        bool done = false;
        gpupr_status status = GPUPR_OK;
        std::string error;              // the failure's message, when status != OK
        gpupr_request_result result{};
    };
    struct Batch {
        std::vector<std::shared_ptr<Request>> reqs;
        std::vector<uint64_t> toff, voff;
        gpupr::DevBuf<int32_t> dT, dN;
        gpupr::DevBuf<double> dV;
        gpupr::DevBuf<uint8_t> dL;
        uint64_t footprint = 0;
        gpupr_status status = GPUPR_OK;
        Clock::time_point t_stage, t_uploaded, t_solve;
    };
    struct Lane {
        int index = 0;
        int max_bps = 0;                // cap on the lane's persistent grid (0 = none)
        cudaStream_t up = nullptr, run = nullptr;
        cudaEvent_t uploaded = nullptr;
        std::deque<std::shared_ptr<Request>> pending;
        std::unique_ptr<Batch> staged;  // uploaded, waiting for the lane's solver
        uint64_t busy_tets = 0;         // tets of the lane's requests submitted and not done
        bool stager_done = false;
        std::thread stager, solver;
    };

    int device = 0;
    uint64_t budget = 0;
    uint32_t max_batch = 0;            // 0 = no limit
    uint64_t split = 0;                // tets from which a request takes the large lane
    gpupr_solve_options opts{};
    bool has_opts = false;
    std::mutex mu;
    std::condition_variable cv;        // any state change; the lanes' threads and waiters
    std::map<uint64_t, std::shared_ptr<Request>> all;
    std::vector<std::unique_ptr<Lane>> lanes;
    uint64_t committed = 0;            // footprint of every batch staged or being solved
    uint64_t next_id = 1;
    bool stopping = false;

    static uint64_t footprint(uint64_t n_tets, uint64_t nv)
    {
        // topology 32 + packed topology 32, labels in/out 2, full_to_free 4,
        // reduced graph + pair sums + base 57, solver workspace 24, free_old 4,
        // segment table 1 (per tet, with free <= tets), vertices 24 per vertex
        return n_tets * 156u + nv * 24u + (1u << 20);
    }

    void stage_loop(Lane& ln);
    void solve_loop(Lane& ln);
    void upload(Lane& ln, Batch& b);
    void solve(Lane& ln, Batch& b);
    // results of a batch: per-request items/status/message when given, else
    // the batch's status for every request
    void publish(Batch& b, const std::vector<gpupr_batch_item>* items,
                 const std::vector<gpupr_status>* status, const std::vector<std::string>* msg,
                 Clock::time_point t_done);
};

void gpupr_server::upload(Lane& ln, Batch& b)
{
    using namespace gpupr;
    const uint32_t G = (uint32_t)b.reqs.size();
    b.toff.assign(G + 1, 0);
    b.voff.assign(G + 1, 0);
    for (uint32_t k = 0; k < G; ++k) {
        b.toff[k + 1] = b.toff[k] + b.reqs[k]->n;
        b.voff[k + 1] = b.voff[k] + b.reqs[k]->nv;
    }
    const uint64_t N = b.toff[G], nv = b.voff[G];
    b.dT = DevBuf<int32_t>(N * 4u, ln.up);
    b.dN = DevBuf<int32_t>(N * 4u, ln.up);
    b.dL = DevBuf<uint8_t>(N, ln.up);
    b.dV = DevBuf<double>(nv * 3u, ln.up);
    for (uint32_t k = 0; k < G; ++k) {
        const Request& r = *b.reqs[k];
        if (!r.n) continue;
        host_to_device(b.dT.p + b.toff[k] * 4u, r.T, r.n * 16u, ln.up);
        host_to_device(b.dN.p + b.toff[k] * 4u, r.Nb, r.n * 16u, ln.up);
        host_to_device(b.dL.p + b.toff[k], r.L, r.n, ln.up);
        host_to_device(b.dV.p + b.voff[k] * 3u, r.V, r.nv * 24u, ln.up);
    }
    GPUPR_CUDA(cudaEventRecord(ln.uploaded, ln.up));
    // the caller's host arrays are read once the copies are done; waiting
    // here also keeps the event free for the lane's next batch
    GPUPR_CUDA(cudaEventSynchronize(ln.uploaded));
}

void gpupr_server::solve(Lane& ln, Batch& b)
{
    using namespace gpupr;
    const uint32_t G = (uint32_t)b.reqs.size();
    std::vector<gpupr_batch_item> items(G);
    std::vector<gpupr_status> status(G, GPUPR_OK);
    std::vector<std::string> msg(G);
    cudaStream_t run = ln.run;
    // cuts requests [k0, k0 + cnt) as one batch; labels straight to their callers
    auto cut = [&](uint32_t k0, uint32_t cnt) {
        std::vector<uint64_t> toff(cnt + 1), voff(cnt + 1);
        for (uint32_t k = 0; k <= cnt; ++k) {
            toff[k] = b.toff[k0 + k] - b.toff[k0];
            voff[k] = b.voff[k0 + k] - b.voff[k0];
        }
        const uint64_t N = toff[cnt];
        gpupr_cut_stats st{};
        DevBuf<uint8_t> dout(N, run);
        run_graph_cut_batch(cnt, toff.data(), voff.data(), b.dV.p + b.voff[k0] * 3u, 1,
                            b.dT.p + b.toff[k0] * 4u, b.dN.p + b.toff[k0] * 4u, b.dL.p + b.toff[k0], 1,
                            b.reqs[k0]->fill_T, has_opts ? &opts : nullptr, dout.p, 1, run,
                            items.data() + k0, &st, ln.max_bps);
        for (uint32_t k = 0; k < cnt; ++k)
            device_to_host(b.reqs[k0 + k]->out, dout.p + toff[k], b.reqs[k0 + k]->n, run);
        GPUPR_CUDA(cudaStreamSynchronize(run));
    };
    auto guarded_cut = [&](uint32_t k0, uint32_t cnt) -> bool {
        gpupr_status s0 = GPUPR_OK;
        std::string m;
        try {
            cut(k0, cnt);
            return true;
        } catch (const Error& e) {
            s0 = e.status;
            m = e.msg;
        } catch (...) {
            s0 = GPUPR_ERR_CUDA;
            m = "unknown failure";
        }
        cudaStreamSynchronize(run);
        cudaGetLastError();
        for (uint32_t k = k0; k < k0 + cnt; ++k) {
            status[k] = s0;
            msg[k] = m;
        }
        return false;
    };
    // one bad request must not fail the others: when the batch fails, every
    // request is cut alone and keeps its own result or error
    if (!guarded_cut(0, G) && G > 1)
        for (uint32_t k = 0; k < G; ++k) {
            status[k] = GPUPR_OK;
            msg[k].clear();
            guarded_cut(k, 1);
        }
    // the staged buffers were written on the upload stream and read on this
    // one, whose work is complete: release them now
    b.dT.reset();
    b.dN.reset();
    b.dL.reset();
    b.dV.reset();
    publish(b, &items, &status, &msg, Clock::now());
}

void gpupr_server::publish(Batch& b, const std::vector<gpupr_batch_item>* items,
                           const std::vector<gpupr_status>* status,
                           const std::vector<std::string>* msg, Clock::time_point t_done)
{
    const uint32_t G = (uint32_t)b.reqs.size();
    auto ms = [](Clock::time_point a, Clock::time_point z) {
        return z > a ? std::chrono::duration<double, std::milli>(z - a).count() : 0.0;
    };
    std::lock_guard<std::mutex> lk(mu);
    for (uint32_t k = 0; k < G; ++k) {
        auto& r = *b.reqs[k];
        r.status = status ? (*status)[k] : b.status;
        if (r.status != GPUPR_OK) r.error = msg ? (*msg)[k] : std::string(gpupr_status_string(r.status));
        if (items && r.status == GPUPR_OK) {
            r.result.adjusted_flow = (*items)[k].adjusted_flow;
            r.result.raw_flow = (*items)[k].raw_flow;
            r.result.free_n = (*items)[k].free_n;
        }
        r.result.id = r.id;
        r.result.status = r.status;
        r.result.n_tets = r.n;
        r.result.batch_size = (int32_t)G;
        r.result.queue_ms = ms(r.t_submit, r.t_start);
        r.result.upload_ms = ms(b.t_stage, b.t_uploaded);
        r.result.solve_ms = ms(b.t_solve, t_done);
        r.result.latency_ms = ms(r.t_submit, t_done);
        r.result.lane = r.lane;
        if (!r.done) lanes[(size_t)r.lane]->busy_tets -= r.n;
        r.done = true;
    }
    cv.notify_all();
}

void gpupr_server::stage_loop(Lane& ln)
{
    cudaSetDevice(device);
    for (;;) {
        auto b = std::make_unique<Batch>();
        {
            std::unique_lock<std::mutex> lk(mu);
            // a request is taken only when the lane's handoff slot is free and
            // it fits next to every batch staged or solving on either lane
            cv.wait(lk, [&] {
                if (stopping && ln.pending.empty()) return true;
                if (ln.staged || ln.pending.empty()) return false;
                return footprint(ln.pending.front()->n, ln.pending.front()->nv) + committed <= budget;
            });
            if (ln.pending.empty()) {
                ln.stager_done = true;
                cv.notify_all();
                return;
            }
            const double fill = ln.pending.front()->fill_T;
            for (auto it = ln.pending.begin(); it != ln.pending.end();) {
                const uint64_t f = footprint((*it)->n, (*it)->nv);
                if (max_batch && b->reqs.size() >= max_batch) break;
                if ((*it)->fill_T == fill && b->footprint + f + committed <= budget) {
                    b->footprint += f;
                    (*it)->t_start = Clock::now();
                    b->reqs.push_back(*it);
                    it = ln.pending.erase(it);
                } else {
                    ++it;
                }
            }
            committed += b->footprint;   // held until the lane's solver is done with it
        }
        b->t_stage = Clock::now();
        try {
            upload(ln, *b);
            b->t_uploaded = Clock::now();
        } catch (const gpupr::Error& e) {
            b->status = e.status;
        } catch (...) {
            b->status = GPUPR_ERR_CUDA;
        }
        if (b->status != GPUPR_OK) {
            cudaStreamSynchronize(ln.up);
            cudaGetLastError();
            b->dT.reset();
            b->dN.reset();
            b->dL.reset();
            b->dV.reset();
            publish(*b, nullptr, nullptr, nullptr, Clock::now());
            std::lock_guard<std::mutex> lk(mu);
            committed -= b->footprint;
            cv.notify_all();
            continue;
        }
        std::lock_guard<std::mutex> lk(mu);
        ln.staged = std::move(b);
        cv.notify_all();
    }
}

void gpupr_server::solve_loop(Lane& ln)
{
    cudaSetDevice(device);
    for (;;) {
        std::unique_ptr<Batch> b;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return ln.staged || ln.stager_done; });
            if (!ln.staged) return;
            b = std::move(ln.staged);
            b->t_solve = Clock::now();
            cv.notify_all();
        }
        solve(ln, *b);
        std::lock_guard<std::mutex> lk(mu);
        committed -= b->footprint;
        cv.notify_all();
    }
}

namespace {

void destroy_lane(gpupr_server::Lane& ln)
{
    if (ln.uploaded) cudaEventDestroy(ln.uploaded);
    if (ln.up) cudaStreamDestroy(ln.up);
    if (ln.run) cudaStreamDestroy(ln.run);
    ln.uploaded = nullptr;
    ln.up = ln.run = nullptr;
}

}  // namespace

extern "C" {

gpupr_status gpupr_server_create_lanes(uint64_t hbm_budget_bytes, uint32_t max_batch,
                                       const gpupr_solve_options* options, uint64_t split_tets,
                                       gpupr_server** server)
{
    if (!server) return GPUPR_ERR_INVALID_ARGUMENT;
    *server = nullptr;
    auto* sv = new (std::nothrow) gpupr_server();
    if (!sv) return GPUPR_ERR_OUT_OF_MEMORY;
    if (cudaGetDevice(&sv->device) != cudaSuccess) {
        cudaGetLastError();
        delete sv;
        return GPUPR_ERR_CUDA;
    }
    // two lanes only when both capped grids fit on the device together
    int occ = 0;
    try {
        occ = gpupr::persistent_blocks_per_sm();
    } catch (const gpupr::Error& e) {
        gpupr::set_last_error(e.msg);
        delete sv;
        return e.status;
    }
    const int nl = (split_tets && occ >= 2) ? 2 : 1;
    sv->split = nl == 2 ? split_tets : 0;
    for (int k = 0; k < nl; ++k) {
        auto ln = std::make_unique<gpupr_server::Lane>();
        ln->index = k;
        ln->max_bps = nl == 1 ? 0 : (k == 0 ? 1 : occ - 1);
        if (cudaStreamCreateWithFlags(&ln->up, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&ln->run, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ln->uploaded, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            destroy_lane(*ln);
            for (auto& l : sv->lanes) destroy_lane(*l);
            delete sv;
            return GPUPR_ERR_CUDA;
        }
        sv->lanes.push_back(std::move(ln));
    }
    sv->budget = hbm_budget_bytes ? hbm_budget_bytes : (160ull << 30);
    sv->max_batch = max_batch;
    if (options) {
        sv->opts = *options;
        sv->has_opts = true;
    }
    for (auto& l : sv->lanes) {
        gpupr_server::Lane* lp = l.get();
        lp->stager = std::thread([sv, lp] { sv->stage_loop(*lp); });
        lp->solver = std::thread([sv, lp] { sv->solve_loop(*lp); });
    }
    *server = sv;
    return GPUPR_OK;
}

gpupr_status gpupr_server_create(uint64_t hbm_budget_bytes, uint32_t max_batch,
                                 const gpupr_solve_options* options, gpupr_server** server)
{
    return gpupr_server_create_lanes(hbm_budget_bytes, max_batch, options, 2000000ull, server);
}

gpupr_status gpupr_server_submit(gpupr_server* sv, const double* vertices, uint64_t n_vertices,
                                 const int32_t* tets, const int32_t* neighbors,
                                 const uint8_t* labels, uint64_t n_tets, double fill_T,
                                 uint8_t* out_labels, uint64_t* request_id)
{
    if (!sv || !request_id || (n_tets && (!tets || !neighbors || !labels || !out_labels)) ||
        (n_vertices && !vertices)) {
        gpupr::set_last_error("gpupr_server_submit: NULL argument");
        return GPUPR_ERR_INVALID_ARGUMENT;
    }
    if (gpupr_server::footprint(n_tets, n_vertices) > sv->budget) {
        gpupr::set_last_error("request footprint exceeds the server's HBM budget");
        return GPUPR_ERR_OUT_OF_MEMORY;
    }
    auto r = std::make_shared<gpupr_server::Request>();
    r->V = vertices;
    r->T = tets;
    r->Nb = neighbors;
    r->L = labels;
    r->out = out_labels;
    r->nv = n_vertices;
    r->n = n_tets;
    r->fill_T = fill_T;
    r->lane = (sv->split && n_tets >= sv->split) ? 1 : 0;
    r->t_submit = gpupr_server::Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stopping) {
            gpupr::set_last_error("the server is shutting down");
            return GPUPR_ERR_INVALID_ARGUMENT;
        }
        // a small request spills to an idle large lane while the small lane is busy
        if (r->lane == 0 && sv->lanes.size() == 2 && sv->lanes[0]->busy_tets > 0 &&
            sv->lanes[1]->busy_tets == 0)
            r->lane = 1;
        sv->lanes[(size_t)r->lane]->busy_tets += r->n;
        r->id = sv->next_id++;
        sv->all[r->id] = r;
        sv->lanes[(size_t)r->lane]->pending.push_back(r);
        *request_id = r->id;
    }
    sv->cv.notify_all();
    return GPUPR_OK;
}

gpupr_status gpupr_server_wait(gpupr_server* sv, uint64_t request_id, double timeout_s,
                               gpupr_request_result* result)
{
    if (!sv) return GPUPR_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->all.find(request_id);
    if (it == sv->all.end()) {
        gpupr::set_last_error("unknown or already read request id");
        return GPUPR_ERR_INVALID_ARGUMENT;
    }
    auto r = it->second;
    const auto limit = std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
    if (!sv->cv.wait_for(lk, limit, [&] { return r->done; })) {
        gpupr::set_last_error("request not finished within the timeout");
        return GPUPR_ERR_TIMEOUT;
    }
    if (r->status != GPUPR_OK) gpupr::set_last_error(r->error);
    if (result) *result = r->result;
    sv->all.erase(it);   // the result is read out: release it
    return r->status;
}

gpupr_status gpupr_server_destroy(gpupr_server* sv)
{
    if (!sv) return GPUPR_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stopping = true;
    }
    sv->cv.notify_all();
    for (auto& l : sv->lanes) {
        if (l->stager.joinable()) l->stager.join();
        if (l->solver.joinable()) l->solver.join();
    }
    for (auto& l : sv->lanes) destroy_lane(*l);
    delete sv;
    return GPUPR_OK;
}

}  // extern "C"
