// server.cu -- continuous-batching serving loop for graph cuts.
//
// Clients submit cut requests (one cell graph each, host arrays) at any time;
// the server borrows the arrays (no host copy) until the request is done and
// writes the labels straight into the caller's output array.  Two threads:
//
//   stager  admits pending requests in arrival order while their estimated
//           device footprint fits the budget left by the batch on the GPU
//           (one batch shares fill_T), copies each request's arrays into the
//           packed device batch on its own stream, and hands the batch over
//           (one staged batch at most);
//   solver  cuts the staged batch as one reduced graph (run_graph_cut_batch:
//           one build, one solve, per-graph flows), copies each request's
//           labels out and publishes the results.
//
// So the upload of batch k+1 overlaps the solve of batch k, requests that
// arrive while a batch runs join the next one, and the GPU never waits for
// a full batch.  Results are exact: the cut of a graph does not depend on
// what else is in its batch.
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

    int device = 0;
    uint64_t budget = 0;
    uint32_t max_batch = 0;            // 0 = no limit
    gpupr_solve_options opts{};
    bool has_opts = false;
    cudaStream_t up = nullptr, run = nullptr;
    cudaEvent_t uploaded = nullptr;
    std::mutex mu;
    std::condition_variable cv;        // any state change; both threads and waiters
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> all;
    std::unique_ptr<Batch> staged;     // uploaded, waiting for the solver
    uint64_t solving_footprint = 0;    // footprint of the batch on the solver
    uint64_t next_id = 1;
    bool stopping = false, stager_done = false;
    std::thread stager, solver;

    static uint64_t footprint(uint64_t n_tets, uint64_t nv)
    {
        // topology 32 + packed topology 32, labels in/out 2, full_to_free 4,
        // reduced graph + base 41, solver workspace 24, free_old 4 (per tet,
        // with free <= tets), vertices 24 per vertex
        return n_tets * 139u + nv * 24u + (1u << 20);
    }

    void stage_loop();
    void solve_loop();
    void upload(Batch& b);
    void solve(Batch& b);
    // results of a batch: per-request items/status/message when given, else
    // the batch's status for every request
    void publish(Batch& b, const std::vector<gpupr_batch_item>* items,
                 const std::vector<gpupr_status>* status, const std::vector<std::string>* msg,
                 Clock::time_point t_done);
};

void gpupr_server::upload(Batch& b)
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
    b.dT = DevBuf<int32_t>(N * 4u, up);
    b.dN = DevBuf<int32_t>(N * 4u, up);
    b.dL = DevBuf<uint8_t>(N, up);
    b.dV = DevBuf<double>(nv * 3u, up);
    for (uint32_t k = 0; k < G; ++k) {
        const Request& r = *b.reqs[k];
        if (!r.n) continue;
        host_to_device(b.dT.p + b.toff[k] * 4u, r.T, r.n * 16u, up);
        host_to_device(b.dN.p + b.toff[k] * 4u, r.Nb, r.n * 16u, up);
        host_to_device(b.dL.p + b.toff[k], r.L, r.n, up);
        host_to_device(b.dV.p + b.voff[k] * 3u, r.V, r.nv * 24u, up);
    }
    GPUPR_CUDA(cudaEventRecord(uploaded, up));
    // the caller's host arrays are read once the copies are done; waiting
    // here also keeps the event free for the next batch
    GPUPR_CUDA(cudaEventSynchronize(uploaded));
}

void gpupr_server::solve(Batch& b)
{
    using namespace gpupr;
    const uint32_t G = (uint32_t)b.reqs.size();
    std::vector<gpupr_batch_item> items(G);
    std::vector<gpupr_status> status(G, GPUPR_OK);
    std::vector<std::string> msg(G);
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
                            items.data() + k0, &st);
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
        r.done = true;
    }
    cv.notify_all();
}

void gpupr_server::stage_loop()
{
    cudaSetDevice(device);
    for (;;) {
        auto b = std::make_unique<Batch>();
        {
            std::unique_lock<std::mutex> lk(mu);
            // a request is taken only when the handoff slot is free and it
            // fits next to the batch on the solver
            cv.wait(lk, [&] {
                if (stopping && pending.empty()) return true;
                if (staged || pending.empty()) return false;
                return footprint(pending.front()->n, pending.front()->nv) + solving_footprint <= budget;
            });
            if (pending.empty()) {
                stager_done = true;
                cv.notify_all();
                return;
            }
            const double fill = pending.front()->fill_T;
            for (auto it = pending.begin(); it != pending.end();) {
                const uint64_t f = footprint((*it)->n, (*it)->nv);
                if (max_batch && b->reqs.size() >= max_batch) break;
                if ((*it)->fill_T == fill && b->footprint + f + solving_footprint <= budget) {
                    b->footprint += f;
                    (*it)->t_start = Clock::now();
                    b->reqs.push_back(*it);
                    it = pending.erase(it);
                } else {
                    ++it;
                }
            }
        }
        b->t_stage = Clock::now();
        try {
            upload(*b);
            b->t_uploaded = Clock::now();
        } catch (const gpupr::Error& e) {
            b->status = e.status;
        } catch (...) {
            b->status = GPUPR_ERR_CUDA;
        }
        if (b->status != GPUPR_OK) {
            cudaStreamSynchronize(up);
            cudaGetLastError();
            b->dT.reset();
            b->dN.reset();
            b->dL.reset();
            b->dV.reset();
            publish(*b, nullptr, nullptr, nullptr, Clock::now());
            continue;
        }
        std::lock_guard<std::mutex> lk(mu);
        staged = std::move(b);
        cv.notify_all();
    }
}

void gpupr_server::solve_loop()
{
    cudaSetDevice(device);
    for (;;) {
        std::unique_ptr<Batch> b;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return staged || stager_done; });
            if (!staged) return;
            b = std::move(staged);
            b->t_solve = Clock::now();
            solving_footprint = b->footprint;
            cv.notify_all();
        }
        solve(*b);
        std::lock_guard<std::mutex> lk(mu);
        solving_footprint = 0;
        cv.notify_all();
    }
}

extern "C" {

gpupr_status gpupr_server_create(uint64_t hbm_budget_bytes, uint32_t max_batch,
                                 const gpupr_solve_options* options, gpupr_server** server)
{
    if (!server) return GPUPR_ERR_INVALID_ARGUMENT;
    *server = nullptr;
    auto* sv = new (std::nothrow) gpupr_server();
    if (!sv) return GPUPR_ERR_OUT_OF_MEMORY;
    if (cudaGetDevice(&sv->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sv->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sv->run, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sv->uploaded, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (sv->uploaded) cudaEventDestroy(sv->uploaded);
        if (sv->up) cudaStreamDestroy(sv->up);
        if (sv->run) cudaStreamDestroy(sv->run);
        delete sv;
        return GPUPR_ERR_CUDA;
    }
    sv->budget = hbm_budget_bytes ? hbm_budget_bytes : (160ull << 30);
    sv->max_batch = max_batch;
    if (options) {
        sv->opts = *options;
        sv->has_opts = true;
    }
    sv->stager = std::thread([sv] { sv->stage_loop(); });
    sv->solver = std::thread([sv] { sv->solve_loop(); });
    *server = sv;
    return GPUPR_OK;
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
    r->t_submit = gpupr_server::Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stopping) {
            gpupr::set_last_error("the server is shutting down");
            return GPUPR_ERR_INVALID_ARGUMENT;
        }
        r->id = sv->next_id++;
        sv->all[r->id] = r;
        sv->pending.push_back(r);
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
    if (sv->stager.joinable()) sv->stager.join();
    if (sv->solver.joinable()) sv->solver.join();
    if (sv->uploaded) cudaEventDestroy(sv->uploaded);
    if (sv->up) cudaStreamDestroy(sv->up);
    if (sv->run) cudaStreamDestroy(sv->run);
    delete sv;
    return GPUPR_OK;
}

}  // extern "C"
