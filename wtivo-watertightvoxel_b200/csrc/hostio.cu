// hostio.cu -- copies between PAGEABLE host arrays and the device.
//
// The drop-in boundary takes numpy arrays (vertices, labels in; labels out),
// and the serving loop takes whole graphs from host memory.  A plain
// cudaMemcpyAsync from pageable memory goes through the driver's own staging
// at the speed of one host thread.  Here each copy is cut into chunks that
// rotate through a few pinned staging buffers: a small pool of host threads
// copies chunk c+1 between the caller's array and a staging buffer while the
// DMA engine moves chunk c, so the copy runs near the PCIe rate instead of
// one core's memcpy rate.  Pinned source/destination arrays skip the staging.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "gpupr_internal.cuh"

namespace gpupr {
namespace {

constexpr size_t kChunk = 8u << 20;     // bytes per staging buffer
constexpr int kSlots = 4;               // staging buffers per direction and device
constexpr size_t kDirect = 1u << 20;    // below this, the driver's own path

// A fixed set of host worker threads that run the parts of one job (a
// memcpy or a row gather) in parallel; the calling thread takes parts too.
// Each job is its own object that workers pick up under the pool mutex, so a
// worker can never take a part of a later job by mistake.
class CopyPool {
public:
    CopyPool()
    {
        int n = 8;
        if (const char* e = std::getenv("GPUPR_COPY_THREADS")) n = std::atoi(e);
        const unsigned hw = std::thread::hardware_concurrency();
        if (hw) n = std::min<int>(n, (int)hw / 2);
        n = std::max(0, std::min(n, 32));
        for (int i = 0; i < n; ++i) workers_.emplace_back([this] { work(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    int threads() const { return (int)workers_.size() + 1; }

    // Runs fn(0..parts-1), returns when every part is done.
    void run(int parts, std::function<void(int)> fn)
    {
        if (parts <= 1 || workers_.empty()) {
            for (int p = 0; p < parts; ++p) fn(p);
            return;
        }
        auto job = std::make_shared<Job>();
        job->fn = std::move(fn);
        job->parts = parts;
        job->left = parts;
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = job;
            ++gen_;
        }
        cv_.notify_all();
        job->run();
        std::unique_lock<std::mutex> lk(job->mu);
        job->cv.wait(lk, [&] { return job->left == 0; });
    }

    void copy(void* dst, const void* src, size_t n)
    {
        const int parts = (int)std::min<size_t>(threads(), std::max<size_t>(1, n / (1u << 20)));
        const size_t per = (n + parts - 1) / parts;
        char* d = static_cast<char*>(dst);
        const char* s = static_cast<const char*>(src);
        run(parts, [=](int p) {
            const size_t b = (size_t)p * per, e = std::min(n, b + per);
            if (b < e) std::memcpy(d + b, s + b, e - b);
        });
    }

private:
    struct Job {
        std::function<void(int)> fn;
        int parts = 0;
        std::atomic<int> next{0};
        int left = 0;
        std::mutex mu;
        std::condition_variable cv;
        void run()
        {
            for (;;) {
                const int p = next.fetch_add(1);
                if (p >= parts) return;
                fn(p);
                std::lock_guard<std::mutex> lk(mu);
                if (--left == 0) cv.notify_all();
            }
        }
    };
    void work()
    {
        uint64_t seen = 0;
        for (;;) {
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                job = job_;
            }
            if (job) job->run();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::shared_ptr<Job> job_;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

CopyPool& copy_pool()
{
    static CopyPool* p = new CopyPool();   // lives for the process
    return *p;
}

struct Staging {
    std::mutex mu;
    char* pin = nullptr;
    cudaEvent_t ev[kSlots] = {};
    bool pending[kSlots] = {};
    bool ok = false;
};

// Staging sets per device and direction (0 = to device, 1 = to host) that
// host threads can hold at the same time, so that copies issued by
// different threads (the server's two lanes, each uploading its own batch)
// run side by side instead of queueing on one set; each set is kSlots x
// kChunk pinned bytes, made on first use with its device current.
constexpr int kSets = 3;

// A staging set held by one copy until the lease goes out of scope.
struct StagingLease {
    Staging* st;
    std::unique_lock<std::mutex> lk;
};

// Takes a staging set of the current device for direction dir that no other
// copy holds; makes one while there are fewer than kSets, else waits for the
// first set.
StagingLease staging(int dir)
{
    static std::mutex mu;
    static std::map<std::pair<int, int>, std::vector<std::unique_ptr<Staging>>> all;
    int dev = 0;
    GPUPR_CUDA(cudaGetDevice(&dev));
    Staging* first = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto& sets = all[{dev, dir}];
        for (auto& s : sets) {
            std::unique_lock<std::mutex> l(s->mu, std::try_to_lock);
            if (l.owns_lock()) return {s.get(), std::move(l)};
        }
        if ((int)sets.size() < kSets) {
            auto s = std::make_unique<Staging>();
            GPUPR_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s->pin), kChunk * kSlots, cudaHostAllocPortable));
            for (int i = 0; i < kSlots; ++i)
                GPUPR_CUDA(cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming));
            s->ok = true;
            std::unique_lock<std::mutex> l(s->mu);
            Staging* p = s.get();
            sets.push_back(std::move(s));
            return {p, std::move(l)};
        }
        first = sets.front().get();
    }
    return {first, std::unique_lock<std::mutex>(first->mu)};
}

// Waits for the copies a previous call left in flight (after an error, or
// the last chunks of a host-to-device copy) before the buffers are reused.
void settle(Staging& st)
{
    for (int k = 0; k < kSlots; ++k)
        if (st.pending[k]) {
            GPUPR_CUDA(cudaEventSynchronize(st.ev[k]));
            st.pending[k] = false;
        }
}

bool is_pinned(const void* p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

void host_to_device(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s)
{
    if (!bytes) return;
    if (bytes < kDirect || is_pinned(h_src)) {
        GPUPR_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    StagingLease lease = staging(0);
    Staging& st = *lease.st;
    settle(st);
    const char* src = static_cast<const char*>(h_src);
    char* dst = static_cast<char*>(d_dst);
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    for (size_t c = 0; c < nch; ++c) {
        const int k = (int)(c % kSlots);
        const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
        char* pin = st.pin + (size_t)k * kChunk;
        if (st.pending[k]) GPUPR_CUDA(cudaEventSynchronize(st.ev[k]));
        copy_pool().copy(pin, src + off, len);
        GPUPR_CUDA(cudaMemcpyAsync(dst + off, pin, len, cudaMemcpyHostToDevice, s));
        GPUPR_CUDA(cudaEventRecord(st.ev[k], s));
        st.pending[k] = true;
    }
}

void device_to_host(void* h_dst, const void* d_src, size_t bytes, cudaStream_t s)
{
    if (!bytes) return;
    if (bytes < kDirect || is_pinned(h_dst)) {
        GPUPR_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, s));
        GPUPR_CUDA(cudaStreamSynchronize(s));
        return;
    }
    StagingLease lease = staging(1);
    Staging& st = *lease.st;
    settle(st);
    const char* src = static_cast<const char*>(d_src);
    char* dst = static_cast<char*>(h_dst);
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t c) {
        const int k = (int)(c % kSlots);
        const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
        GPUPR_CUDA(cudaMemcpyAsync(st.pin + (size_t)k * kChunk, src + off, len,
                                   cudaMemcpyDeviceToHost, s));
        GPUPR_CUDA(cudaEventRecord(st.ev[k], s));
        st.pending[k] = true;
    };
    for (size_t c = 0; c < std::min<size_t>(nch, kSlots); ++c) issue(c);
    for (size_t c = 0; c < nch; ++c) {
        const int k = (int)(c % kSlots);
        const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
        GPUPR_CUDA(cudaEventSynchronize(st.ev[k]));
        copy_pool().copy(dst + off, st.pin + (size_t)k * kChunk, len);
        st.pending[k] = false;
        if (c + kSlots < nch) issue(c + kSlots);
    }
}

// Nx4 integer topology (int32 or int64 elements, any byte strides, e.g. a
// Fortran-ordered matrix) -> contiguous int32 Nx4 on the device.  Rows are
// gathered chunk by chunk into the pinned staging by the host pool while the
// previous chunk is in flight; int64 values are narrowed the way numpy's
// astype(int32) narrows them (low 32 bits).
void upload_topology(int32_t* d_out, const void* host, uint64_t rows, int64_t row_stride,
                     int64_t col_stride, int elem_bytes, cudaStream_t s)
{
    if (!rows) return;
    if (elem_bytes == 4 && row_stride == 16 && col_stride == 4) {
        host_to_device(d_out, host, rows * 16u, s);
        return;
    }
    const char* base = static_cast<const char*>(host);
    StagingLease lease = staging(0);
    Staging& st = *lease.st;
    settle(st);
    const uint64_t per_chunk = kChunk / 16u;
    const uint64_t nch = (rows + per_chunk - 1) / per_chunk;
    CopyPool& pool = copy_pool();
    for (uint64_t c = 0; c < nch; ++c) {
        const int k = (int)(c % kSlots);
        const uint64_t r0 = c * per_chunk, r1 = std::min(rows, r0 + per_chunk);
        int32_t* pin = reinterpret_cast<int32_t*>(st.pin + (size_t)k * kChunk);
        if (st.pending[k]) GPUPR_CUDA(cudaEventSynchronize(st.ev[k]));
        const int parts = std::max(1, std::min(pool.threads(), (int)((r1 - r0) / 16384u)));
        const uint64_t per = (r1 - r0 + parts - 1) / parts;
        pool.run(parts, [=](int p) {
            const uint64_t a = r0 + (uint64_t)p * per, z = std::min(r1, a + per);
            for (uint64_t r = a; r < z; ++r) {
                const char* row = base + (int64_t)r * row_stride;
                int32_t* o = pin + (r - r0) * 4u;
                for (int j = 0; j < 4; ++j) {
                    const char* e = row + (int64_t)j * col_stride;
                    if (elem_bytes == 8) {
                        int64_t v;
                        std::memcpy(&v, e, 8);
                        o[j] = (int32_t)(uint32_t)(uint64_t)v;
                    } else {
                        std::memcpy(&o[j], e, 4);
                    }
                }
            }
        });
        GPUPR_CUDA(cudaMemcpyAsync(d_out + r0 * 4u, pin, (r1 - r0) * 16u, cudaMemcpyHostToDevice, s));
        GPUPR_CUDA(cudaEventRecord(st.ev[k], s));
        st.pending[k] = true;
    }
}

namespace {

struct ThreadRes {
    int device = -1;
    Ctl* ctl = nullptr;
    cudaEvent_t ev[8] = {};
    ~ThreadRes()
    {
        if (ctl) cudaFreeHost(ctl);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

ThreadRes& thread_res()
{
    thread_local std::vector<std::unique_ptr<ThreadRes>> all;
    int dev = 0;
    GPUPR_CUDA(cudaGetDevice(&dev));
    for (auto& r : all)
        if (r->device == dev) return *r;
    auto r = std::make_unique<ThreadRes>();
    r->device = dev;
    GPUPR_CUDA(cudaMallocHost(reinterpret_cast<void**>(&r->ctl), sizeof(Ctl)));
    for (cudaEvent_t& e : r->ev) GPUPR_CUDA(cudaEventCreate(&e));
    all.push_back(std::move(r));
    return *all.back();
}

}  // namespace

Ctl* pinned_ctl() { return thread_res().ctl; }

cudaEvent_t timing_event(int slot) { return thread_res().ev[slot & 7]; }

}  // namespace gpupr
