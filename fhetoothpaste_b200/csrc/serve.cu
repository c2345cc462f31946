// Serving loop for blind-rotation (bootstrap) requests of mixed parameter sets.
//
// One scheduler thread per server owns all device work. Clients submit single
// rotations (an LWE, a test polynomial, a result buffer) for a registered
// parameter set; the scheduler batches what is pending per set into one of
// that set's launch buffers and launches the batched rotation on the buffer's
// own stream. Each set has `buffers` launch buffers of `max_batch` slots, all
// reserved at registration, so admission is bounded by the device memory set
// aside for accumulators, inputs and results: requests that arrive while
// others are on the GPU wait in the queue only until a buffer frees, then run
// while the earlier launches are still in flight (different streams, so their
// blocks overlap on the SMs). Keys and tables stay resident in the contexts.
// A request's result depends only on its own inputs: batching changes which
// launch, slot and kernel (one or two blocks per rotation, chosen per launch by
// its size) it runs in, never the words it produces.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "toothpaste_gpu.h"
#include "br_launch.h"
#include "serve_policy.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket;
    uint32_t set;
    uint64_t bytes;             // device bytes reserved for it until it completes
    const uint64_t* lwe;
    const uint64_t* acc;
    uint64_t* result;
    Clock::time_point t_submit;
};

struct LaunchBuffer {
    uint64_t* d_lwe = nullptr;
    uint64_t* d_acc = nullptr;
    uint64_t* d_res = nullptr;
    uint64_t* h_lwe = nullptr;  // pinned staging
    uint64_t* h_acc = nullptr;
    uint64_t* h_res = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Request> reqs;  // in flight when non-empty
    uint32_t blocks = 0;        // thread blocks of the launch in flight
};

struct Set {
    tp_br_ctx* ctx = nullptr;
    uint32_t N = 0, n = 0;
    uint32_t max_batch = 0;
    int out_coef = 0;
    uint64_t req_bytes = 0;     // device bytes of one request: its LWE, test polynomial and result
    std::vector<LaunchBuffer> bufs;
    std::deque<Request> pending;
};

}  // namespace

struct tp_server {
    int device = 0;
    uint32_t sm_count = 0;
    uint64_t max_queue = 0;
    std::vector<Set> sets;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::atomic<bool> stop{false};
    std::thread worker;
    uint64_t next_ticket = 1;
    uint64_t queued = 0;
    // completion bookkeeping
    std::vector<uint8_t> done_flag;  // by ticket
    std::vector<double> latency_ms;  // completed requests, in completion order
    uint64_t completed = 0, rejected = 0, launches = 0;
    // device-memory admission: requests reserve their device bytes from the budget when
    // admitted and return them when their result is back in host memory
    uint64_t mem_budget = 0;    // 0 until set: the free device memory at tp_server_start
    bool mem_budget_set = false;
    uint64_t mem_in_use = 0;
    uint64_t rejected_memory = 0;
    tp_status worker_status = TP_OK;
    std::string worker_error;
    Clock::time_point t_first, t_last;
};

namespace {

thread_local std::string s_err;

tp_status serr(tp_status s, const std::string& msg) {
    s_err = msg;
    return s;
}

void release_set(Set& s) {
    for (auto& b : s.bufs) {
        cudaFree(b.d_lwe);
        cudaFree(b.d_acc);
        cudaFree(b.d_res);
        cudaFreeHost(b.h_lwe);
        cudaFreeHost(b.h_acc);
        cudaFreeHost(b.h_res);
        if (b.stream) cudaStreamDestroy(b.stream);
        if (b.done) cudaEventDestroy(b.done);
    }
    s.bufs.clear();
}

// Thread blocks of every set's launches still in flight (one block per SM at the
// serving sets' sizes). Called with mu held.
uint64_t blocks_in_flight(const tp_server* srv) {
    uint64_t k = 0;
    for (const auto& s : srv->sets)
        for (const auto& b : s.bufs) k += b.reqs.empty() ? 0u : b.blocks;
    return k;
}

// Launches pending requests of set `s` into free buffers. Called with mu held.
void launch_pending(tp_server* srv, uint32_t si) {
    Set& s = srv->sets[si];
    for (auto& b : s.bufs) {
        if (s.pending.empty()) return;
        if (!b.reqs.empty()) continue;
        const uint32_t take = (uint32_t)std::min<size_t>(s.pending.size(), s.max_batch);
        const uint64_t busy = blocks_in_flight(srv);  // before this buffer takes its requests
        const uint64_t lw = s.n + 1, aw = 2ull * s.N;
        for (uint32_t i = 0; i < take; ++i) {
            Request r = s.pending.front();
            s.pending.pop_front();
            std::memcpy(b.h_lwe + i * lw, r.lwe, lw * 8);
            std::memcpy(b.h_acc + i * aw, r.acc, aw * 8);
            b.reqs.push_back(r);
        }
        srv->queued -= take;
        cudaError_t e = cudaMemcpyAsync(b.d_lwe, b.h_lwe, take * lw * 8, cudaMemcpyHostToDevice, b.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b.d_acc, b.h_acc, take * aw * 8, cudaMemcpyHostToDevice, b.stream);
        // A launch that leaves SMs idle runs each rotation on two SMs (about half
        // the latency); a launch of a full wave or more runs one block per rotation.
        // A launch of a few requests whose four blocks per rotation fit on the SMs
        // the launches in flight leave free (light load) runs on four where the set's
        // four-block kernel fits (15-30% less latency again); under load the
        // four-block form's extra SM-time (1.7x the two-block form's) would slow the
        // other launches, so it is not used.
        const int split = tp::serve_split(take, busy, srv->sm_count, tp::br_concurrency(s.ctx, 4),
                                          tp::br_concurrency(s.ctx, 2));
        // thread blocks (SMs) the launch keeps busy; a ring above 4096 takes a cluster per rotation
        b.blocks = (uint32_t)(tp::serve_blocks(split, take, tp::br_concurrency(s.ctx, split)) *
                              (split == 1 ? (uint64_t)tp::br_cluster_ctas(s.ctx) : 1u));
        tp_status st = e == cudaSuccess ? tp::br_batch_launch(s.ctx, take, b.d_res, b.d_lwe, lw, b.d_acc, aw,
                                                               s.out_coef, b.stream, split)
                                        : TP_ERR_CUDA;
        if (st == TP_OK) e = cudaMemcpyAsync(b.h_res, b.d_res, take * aw * 8, cudaMemcpyDeviceToHost, b.stream);
        if (st == TP_OK && e == cudaSuccess) e = cudaEventRecord(b.done, b.stream);
        if (st != TP_OK || e != cudaSuccess) {
            srv->worker_status = st != TP_OK ? st : TP_ERR_CUDA;
            srv->worker_error = st != TP_OK ? tp_last_error() : cudaGetErrorString(e);
        }
        srv->launches++;
    }
}

// Retires finished launches of every set. Called with mu held.
bool retire_done(tp_server* srv) {
    bool any = false;
    for (auto& s : srv->sets) {
        for (auto& b : s.bufs) {
            if (b.reqs.empty()) continue;
            if (cudaEventQuery(b.done) != cudaSuccess) continue;
            const auto now = Clock::now();
            const uint64_t aw = 2ull * s.N;
            for (size_t i = 0; i < b.reqs.size(); ++i) {
                const Request& r = b.reqs[i];
                std::memcpy(r.result, b.h_res + i * aw, aw * 8);
                srv->done_flag[r.ticket] = 1;
                srv->mem_in_use -= r.bytes;
                srv->latency_ms.push_back(std::chrono::duration<double, std::milli>(now - r.t_submit).count());
                srv->completed++;
            }
            srv->t_last = now;
            b.reqs.clear();
            any = true;
        }
    }
    return any;
}

void worker_loop(tp_server* srv) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lk(srv->mu);
    while (!srv->stop.load()) {
        bool inflight = false;
        for (uint32_t si = 0; si < srv->sets.size(); ++si) launch_pending(srv, si);
        if (retire_done(srv)) srv->cv_done.notify_all();
        for (auto& s : srv->sets)
            for (auto& b : s.bufs) inflight |= !b.reqs.empty();
        if (!inflight && srv->queued == 0) {
            srv->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
            // poll completions at a fine grain without holding the lock
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        }
    }
}

}  // namespace

extern "C" {

tp_status tp_server_create(int device, uint64_t max_queue, tp_server** out) {
    if (!out) return serr(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return serr(TP_ERR_CUDA, "cudaSetDevice failed");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return serr(TP_ERR_CUDA, "cudaDeviceGetAttribute failed");
    auto* srv = new tp_server();
    srv->device = device;
    srv->sm_count = (uint32_t)sms;
    srv->max_queue = max_queue ? max_queue : 1u << 20;
    *out = srv;
    return TP_OK;
}

tp_status tp_server_add_set(tp_server* srv, tp_br_ctx* ctx, uint32_t ring_dim, uint32_t lwe_dim, uint32_t max_batch,
                            uint32_t buffers, int out_coef, uint32_t* set_id) {
    if (!srv || !ctx || !set_id) return serr(TP_ERR_PARAM, "null argument");
    if (max_batch == 0 || buffers == 0) return serr(TP_ERR_PARAM, "max_batch and buffers must be positive");
    if (srv->worker.joinable()) return serr(TP_ERR_STATE, "sets must be added before tp_server_start");
    cudaSetDevice(srv->device);
    Set s;
    s.ctx = ctx;
    s.N = ring_dim;
    s.n = lwe_dim;
    s.max_batch = max_batch;
    s.out_coef = out_coef;
    const uint64_t lw = (uint64_t)lwe_dim + 1, aw = 2ull * ring_dim;
    s.req_bytes = (lw + 2 * aw) * 8;
    const uint64_t per_buf = ((uint64_t)max_batch * lw + 2 * (uint64_t)max_batch * aw) * 8;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if ((uint64_t)buffers * per_buf > free_b)
        return serr(TP_ERR_OOM, "not enough free device memory for the requested launch buffers");
    s.bufs.resize(buffers);
    for (auto& b : s.bufs) {
        cudaError_t e = cudaMalloc(&b.d_lwe, max_batch * lw * 8);
        if (e == cudaSuccess) e = cudaMalloc(&b.d_acc, max_batch * aw * 8);
        if (e == cudaSuccess) e = cudaMalloc(&b.d_res, max_batch * aw * 8);
        if (e == cudaSuccess) e = cudaMallocHost(&b.h_lwe, max_batch * lw * 8);
        if (e == cudaSuccess) e = cudaMallocHost(&b.h_acc, max_batch * aw * 8);
        if (e == cudaSuccess) e = cudaMallocHost(&b.h_res, max_batch * aw * 8);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            release_set(s);
            return serr(e == cudaErrorMemoryAllocation ? TP_ERR_OOM : TP_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    *set_id = (uint32_t)srv->sets.size();
    srv->sets.push_back(std::move(s));
    return TP_OK;
}

tp_status tp_server_set_memory_budget(tp_server* srv, uint64_t bytes) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->mem_budget = bytes;
    srv->mem_budget_set = true;
    return TP_OK;
}

tp_status tp_server_memory(tp_server* srv, uint64_t* budget, uint64_t* in_use, uint64_t* rejected_memory) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (budget) *budget = srv->mem_budget;
    if (in_use) *in_use = srv->mem_in_use;
    if (rejected_memory) *rejected_memory = srv->rejected_memory;
    return TP_OK;
}

tp_status tp_server_start(tp_server* srv) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    if (srv->worker.joinable()) return TP_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (!srv->mem_budget_set) {
            // by default the device memory still free once keys and launch buffers are resident
            size_t free_b = 0, total_b = 0;
            cudaSetDevice(srv->device);
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return serr(TP_ERR_CUDA, "cudaMemGetInfo failed");
            srv->mem_budget = free_b;
            srv->mem_budget_set = true;
        }
    }
    srv->stop = false;
    srv->worker = std::thread(worker_loop, srv);
    return TP_OK;
}

tp_status tp_server_submit(tp_server* srv, uint32_t set_id, const uint64_t* lwe, const uint64_t* acc,
                           uint64_t* result, uint64_t* ticket) {
    if (!srv || !lwe || !acc || !result || !ticket) return serr(TP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (set_id >= srv->sets.size()) return serr(TP_ERR_PARAM, "unknown set");
    if (srv->worker_status != TP_OK) return serr(srv->worker_status, srv->worker_error);
    if (srv->queued >= srv->max_queue) {
        srv->rejected++;
        return serr(TP_ERR_STATE, "queue full: request rejected by admission control");
    }
    const uint64_t bytes = srv->sets[set_id].req_bytes;
    if (srv->mem_budget_set && srv->mem_in_use + bytes > srv->mem_budget) {
        srv->rejected++;
        srv->rejected_memory++;
        return serr(TP_ERR_OOM, "device memory budget exhausted: request rejected by admission control");
    }
    const uint64_t t = srv->next_ticket++;
    if (srv->done_flag.size() <= t) srv->done_flag.resize(std::max<size_t>(2 * srv->done_flag.size(), t + 1), 0);
    srv->mem_in_use += bytes;
    Request r{t, set_id, bytes, lwe, acc, result, Clock::now()};
    if (srv->completed == 0 && srv->queued == 0 && srv->launches == 0) srv->t_first = r.t_submit;
    srv->sets[set_id].pending.push_back(r);
    srv->queued++;
    *ticket = t;
    srv->cv_work.notify_one();
    return TP_OK;
}

tp_status tp_server_wait(tp_server* srv, uint64_t ticket, uint32_t timeout_ms) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    std::unique_lock<std::mutex> lk(srv->mu);
    const bool ok = srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
        return (ticket < srv->done_flag.size() && srv->done_flag[ticket]) || srv->worker_status != TP_OK;
    });
    if (srv->worker_status != TP_OK) return serr(srv->worker_status, srv->worker_error);
    return ok ? TP_OK : serr(TP_ERR_TIMEOUT, "request not finished within the timeout");
}

tp_status tp_server_drain(tp_server* srv, uint32_t timeout_ms) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    std::unique_lock<std::mutex> lk(srv->mu);
    const bool ok = srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
        if (srv->worker_status != TP_OK) return true;
        if (srv->queued) return false;
        for (auto& s : srv->sets)
            for (auto& b : s.bufs)
                if (!b.reqs.empty()) return false;
        return true;
    });
    if (srv->worker_status != TP_OK) return serr(srv->worker_status, srv->worker_error);
    return ok ? TP_OK : serr(TP_ERR_TIMEOUT, "server did not drain within the timeout");
}

// stats: [completed, rejected, launches, seconds first-submit..last-completion,
//         p50, p99, p99.9, max latency in ms]
tp_status tp_server_stats(tp_server* srv, double* stats8) {
    if (!srv || !stats8) return serr(TP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    std::vector<double> l = srv->latency_ms;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min<size_t>(l.size() - 1, (size_t)(q * l.size()))]; };
    stats8[0] = (double)srv->completed;
    stats8[1] = (double)srv->rejected;
    stats8[2] = (double)srv->launches;
    stats8[3] = srv->completed ? std::chrono::duration<double>(srv->t_last - srv->t_first).count() : 0.0;
    stats8[4] = pct(0.50);
    stats8[5] = pct(0.99);
    stats8[6] = pct(0.999);
    stats8[7] = l.empty() ? 0.0 : l.back();
    return TP_OK;
}

tp_status tp_server_reset_stats(tp_server* srv) {
    if (!srv) return serr(TP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->latency_ms.clear();
    srv->completed = srv->rejected = srv->launches = 0;
    srv->rejected_memory = 0;
    return TP_OK;
}

tp_status tp_server_destroy(tp_server* srv) {
    if (!srv) return TP_OK;
    if (srv->worker.joinable()) {
        srv->stop = true;
        srv->cv_work.notify_all();
        srv->worker.join();
    }
    cudaSetDevice(srv->device);
    for (auto& s : srv->sets) {
        for (auto& b : s.bufs)
            if (b.stream) cudaStreamSynchronize(b.stream);
        release_set(s);
    }
    delete srv;
    return TP_OK;
}

const char* tp_server_last_error(void) { return s_err.c_str(); }

// Open-loop load generator: Poisson arrivals at `rate` requests/s for
// `seconds`, set i drawn with probability mix[i]; request inputs are taken
// round-robin from per-set pools (pool_lwe[i]: pool_n[i] rows of n_i+1 words,
// pool_acc[i]: pool_n[i] rows of 2N_i words). Requests the admission control
// rejects are counted, not retried. Returns when every admitted request has
// finished (or after `seconds` + 60 s).
tp_status tp_server_run_poisson(tp_server* srv, double rate, double seconds, const double* mix, uint32_t nsets,
                                const uint64_t* const* pool_lwe, const uint64_t* const* pool_acc,
                                const uint64_t* pool_n, uint64_t seed) {
    if (!srv || !mix || !pool_lwe || !pool_acc || !pool_n) return serr(TP_ERR_PARAM, "null argument");
    if (nsets != srv->sets.size()) return serr(TP_ERR_PARAM, "mix must cover every registered set");
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate);
    std::discrete_distribution<uint32_t> pick(mix, mix + nsets);
    std::vector<std::vector<uint64_t>> results(nsets);
    std::vector<uint64_t> next(nsets, 0);
    const uint64_t cap = (uint64_t)(rate * seconds * 1.2) + 16;
    std::vector<std::vector<uint64_t>> outbuf(nsets);
    for (uint32_t i = 0; i < nsets; ++i) outbuf[i].resize(2ull * srv->sets[i].N * std::min<uint64_t>(cap, 1 << 16));
    const auto t0 = Clock::now();
    double t = 0;
    while (true) {
        t += gap(rng);
        if (t > seconds) break;
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(t));
        std::this_thread::sleep_until(due);
        const uint32_t si = pick(rng);
        const Set& s = srv->sets[si];
        const uint64_t k = next[si]++ % pool_n[si];
        const uint64_t slot = next[si] % (outbuf[si].size() / (2ull * s.N));
        uint64_t ticket;
        tp_server_submit(srv, si, pool_lwe[si] + k * (s.n + 1), pool_acc[si] + k * 2ull * s.N,
                         outbuf[si].data() + slot * 2ull * s.N, &ticket);
    }
    return tp_server_drain(srv, (uint32_t)(60000 + seconds * 1000));
}

}  // extern "C"
