// server.cu -- continuous-batching serving loop for graph cuts.
//
// Clients submit cut requests (one cell graph each, host arrays) at any time.
// One worker thread per server loops:
//   1. admit: take pending requests in arrival order while their estimated
//      device footprint fits the HBM budget (requests of one batch share
//      fill_T; a request alone larger than the budget is refused at submit);
//   2. solve: pack the admitted graphs and cut them as one batch on the GPU
//      (run_graph_cut_batch: one build, one solve, per-graph flows);
//   3. publish: each request's labels and flows become available to wait().
// Requests that arrive while a batch is on the GPU join the next iteration,
// so the GPU never waits for a full batch and small requests are not held
// behind a queue of large ones longer than one iteration.  Results are exact
// (the cut of a graph does not depend on what else is in its batch).
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
#include <thread>
#include <vector>

#include "gpupr_internal.cuh"
#include "wtivo_gpupr.h"

struct gpupr_server {
    using Clock = std::chrono::steady_clock;
    struct Request {
        uint64_t id = 0;
        std::vector<double> V;
        std::vector<int32_t> T, Nb;
        std::vector<uint8_t> L, out;
        double fill_T = 10.0;
        Clock::time_point t_submit, t_start, t_done;
        bool done = false;
        gpupr_status status = GPUPR_OK;
        gpupr_request_result result{};
    };

    int device = 0;
    uint64_t budget = 0;
    gpupr_solve_options opts{};
    bool has_opts = false;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> all;
    uint64_t next_id = 1;
    bool stopping = false;
    std::thread worker;
    uint64_t batches = 0, served = 0;

    static uint64_t footprint(uint64_t n_tets, uint64_t nv)
    {
        // local + packed topology 64, labels in/out 2, full_to_free 4, reduced
        // graph + base 41, solver workspace 24, free_old 4 (per tet, with
        // free <= tets), vertices 24 per vertex
        return n_tets * 139u + nv * 24u + (1u << 20);
    }

    void loop();
    void run_batch(std::vector<std::shared_ptr<Request>>& batch);
};

void gpupr_server::run_batch(std::vector<std::shared_ptr<Request>>& batch)
{
    using namespace gpupr;
    const uint32_t G = (uint32_t)batch.size();
    std::vector<uint64_t> toff(G + 1, 0), voff(G + 1, 0);
    for (uint32_t k = 0; k < G; ++k) {
        toff[k + 1] = toff[k] + batch[k]->L.size();
        voff[k + 1] = voff[k] + batch[k]->V.size() / 3u;
    }
    const uint64_t N = toff[G], nv = voff[G];
    std::vector<double> V(nv * 3u);
    std::vector<int32_t> T(N * 4u), Nb(N * 4u);
    std::vector<uint8_t> L(N), out(N);
    for (uint32_t k = 0; k < G; ++k) {
        const auto& r = *batch[k];
        std::memcpy(V.data() + voff[k] * 3u, r.V.data(), r.V.size() * sizeof(double));
        std::memcpy(T.data() + toff[k] * 4u, r.T.data(), r.T.size() * sizeof(int32_t));
        std::memcpy(Nb.data() + toff[k] * 4u, r.Nb.data(), r.Nb.size() * sizeof(int32_t));
        std::memcpy(L.data() + toff[k], r.L.data(), r.L.size());
    }
    std::vector<gpupr_batch_item> items(G);
    gpupr_cut_stats st{};
    gpupr_status status = GPUPR_OK;
    const auto t0 = Clock::now();
    try {
        DevBuf<int32_t> dT(N * 4u, stream), dN(N * 4u, stream);
        if (N) {
            GPUPR_CUDA(cudaMemcpyAsync(dT.p, T.data(), N * 16u, cudaMemcpyHostToDevice, stream));
            GPUPR_CUDA(cudaMemcpyAsync(dN.p, Nb.data(), N * 16u, cudaMemcpyHostToDevice, stream));
        }
        run_graph_cut_batch(G, toff.data(), voff.data(), V.data(), 0, dT.p, dN.p, L.data(), 0,
                            batch[0]->fill_T, has_opts ? &opts : nullptr, out.data(), 0, stream,
                            items.data(), &st);
    } catch (const Error& e) {
        status = e.status;
    } catch (...) {
        status = GPUPR_ERR_CUDA;
    }
    const auto t1 = Clock::now();
    const double solve_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::lock_guard<std::mutex> lk(mu);
    for (uint32_t k = 0; k < G; ++k) {
        auto& r = *batch[k];
        r.status = status;
        r.t_done = t1;
        if (status == GPUPR_OK) {
            r.out.assign(out.begin() + (long)toff[k], out.begin() + (long)toff[k + 1]);
            r.result.adjusted_flow = items[k].adjusted_flow;
            r.result.raw_flow = items[k].raw_flow;
            r.result.free_n = items[k].free_n;
        }
        r.result.id = r.id;
        r.result.status = status;
        r.result.n_tets = r.L.size();
        r.result.batch_size = G;
        r.result.solve_ms = solve_ms;
        r.result.queue_ms = std::chrono::duration<double, std::milli>(r.t_start - r.t_submit).count();
        r.result.latency_ms = std::chrono::duration<double, std::milli>(t1 - r.t_submit).count();
        std::vector<double>().swap(r.V);
        std::vector<int32_t>().swap(r.T);
        std::vector<int32_t>().swap(r.Nb);
        r.done = true;
    }
    ++batches;
    served += G;
    cv_done.notify_all();
}

void gpupr_server::loop()
{
    cudaSetDevice(device);
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stopping || !pending.empty(); });
            if (stopping && pending.empty()) return;
            uint64_t used = 0;
            const double fill = pending.front()->fill_T;
            for (auto it = pending.begin(); it != pending.end();) {
                auto& r = *it;
                const uint64_t f = footprint(r->L.size(), r->V.size() / 3u);
                if (r->fill_T == fill && (batch.empty() || used + f <= budget)) {
                    used += f;
                    r->t_start = Clock::now();
                    batch.push_back(r);
                    it = pending.erase(it);
                } else {
                    ++it;
                }
            }
        }
        run_batch(batch);
    }
}

extern "C" {

gpupr_status gpupr_server_create(uint64_t hbm_budget_bytes, const gpupr_solve_options* options,
                                 gpupr_server** server)
{
    if (!server) return GPUPR_ERR_INVALID_ARGUMENT;
    *server = nullptr;
    auto* sv = new (std::nothrow) gpupr_server();
    if (!sv) return GPUPR_ERR_OUT_OF_MEMORY;
    if (cudaGetDevice(&sv->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete sv;
        return GPUPR_ERR_CUDA;
    }
    sv->budget = hbm_budget_bytes ? hbm_budget_bytes : (160ull << 30);
    if (options) {
        sv->opts = *options;
        sv->has_opts = true;
    }
    sv->worker = std::thread([sv] { sv->loop(); });
    *server = sv;
    return GPUPR_OK;
}

gpupr_status gpupr_server_submit(gpupr_server* sv, const double* vertices, uint64_t n_vertices,
                                 const int32_t* tets, const int32_t* neighbors,
                                 const uint8_t* labels, uint64_t n_tets, double fill_T,
                                 uint64_t* request_id)
{
    if (!sv || !request_id || (n_tets && (!tets || !neighbors || !labels)) ||
        (n_vertices && !vertices)) {
        gpupr::set_last_error("gpupr_server_submit: NULL argument");
        return GPUPR_ERR_INVALID_ARGUMENT;
    }
    if (gpupr_server::footprint(n_tets, n_vertices) > sv->budget) {
        gpupr::set_last_error("request footprint exceeds the server's HBM budget");
        return GPUPR_ERR_OUT_OF_MEMORY;
    }
    auto r = std::make_shared<gpupr_server::Request>();
    r->V.assign(vertices, vertices + n_vertices * 3u);
    r->T.assign(tets, tets + n_tets * 4u);
    r->Nb.assign(neighbors, neighbors + n_tets * 4u);
    r->L.assign(labels, labels + n_tets);
    r->fill_T = fill_T;
    r->t_submit = gpupr_server::Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stopping) return GPUPR_ERR_INVALID_ARGUMENT;
        r->id = sv->next_id++;
        sv->all[r->id] = r;
        sv->pending.push_back(r);
        *request_id = r->id;
    }
    sv->cv_work.notify_one();
    return GPUPR_OK;
}

gpupr_status gpupr_server_wait(gpupr_server* sv, uint64_t request_id, double timeout_s,
                               uint8_t* out_labels, gpupr_request_result* result)
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
    if (!sv->cv_done.wait_for(lk, limit, [&] { return r->done; })) {
        gpupr::set_last_error("request not finished within the timeout");
        return GPUPR_ERR_TIMEOUT;
    }
    if (r->status != GPUPR_OK) gpupr::set_last_error(gpupr_status_string(r->status));
    if (out_labels && r->status == GPUPR_OK && !r->out.empty())
        std::memcpy(out_labels, r->out.data(), r->out.size());
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
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    if (sv->stream) cudaStreamDestroy(sv->stream);
    delete sv;
    return GPUPR_OK;
}

}  // extern "C"
