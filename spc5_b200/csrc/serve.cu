// serve.cu -- request loop over resident matrices (continuous batching).
//
// Matrices are registered once and stay on the device; registration is
// admitted against an HBM budget that also covers the per-slot staging
// buffers.  A request is y = A_id x for device vectors x (ncols) and y
// (nrows).  One scheduler thread owns `slots` CUDA streams, each with
// column-major staging blocks X (ncols x max_k) and Y (nrows x max_k):
//   * whenever a slot is free and requests are pending, it takes the matrix
//     whose oldest request waits longest, coalesces up to max_k of its
//     requests (copies each x into a column of X), runs one multi-RHS SpMM
//     (spmm.cu, spmm_rows.cu) and copies each column of Y to its request's
//     y; a lone request runs the matrix's SpMV into its own y instead;
//   * requests that arrive while launches are in flight wait for the next
//     free slot and are batched then, so up to `slots` launches overlap on
//     the device and the batch size adapts to the arrival rate;
//   * completion is detected with an event per launch; latency is measured
//     from submit to the host seeing the event complete.
// Every column of the SpMM is bit-identical to a solo SpMV (every SpMV kernel
// gives the same bits), so a request's result does not depend on what it was
// batched with.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "handle.h"

namespace spc5cuda {
namespace {

using Clock = std::chrono::steady_clock;

double now_us() {
    return std::chrono::duration<double, std::micro>(Clock::now().time_since_epoch()).count();
}

struct Request {
    int mat = 0;
    const void* x = nullptr;
    void* y = nullptr;
    double t_submit = 0.0;
    double t_done = 0.0;
    bool done = false;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t event = nullptr;
    Owned X, Y;
    bool busy = false;
    std::vector<long> reqs;
};

}  // namespace
}  // namespace spc5cuda

using namespace spc5cuda;

struct spc5cuda_server {
    spc5cuda_server_config cfg{};
    int device = 0;
    std::vector<spc5cuda_mat*> mats;
    long resident_bytes = 0;
    int max_rows = 0, max_cols = 0;
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_work;   // new request / shutdown
    std::condition_variable cv_done;   // a request completed
    std::unordered_map<int, std::deque<long>> pending;  // per matrix, FIFO
    std::unordered_map<long, Request> reqs;
    long next_id = 1;
    long inflight = 0;  // submitted and not yet completed
    bool stop = false;
    spc5cuda_status error = SPC5CUDA_OK;
    std::thread worker;

    // statistics
    std::vector<double> lat_us;
    long launches = 0;
    long completed = 0;
    long coalesced = 0;  // sum of k over launches
    double t_first = 0.0, t_last = 0.0;

    long slot_bytes(int rows, int cols) const {
        const long vb = cfg.mixed ? 4 : 8;  // x element size
        const long yb = 8;
        return long(cfg.slots) * long(cfg.max_k) * (long(cols) * (cfg.mixed ? vb : yb) + long(rows) * yb);
    }

    void run();
    bool dispatch(Slot& sl);
    bool finish_dispatch(Slot& sl, int k);
    void complete(Slot& sl);
};

void spc5cuda_server::complete(Slot& sl) {
    const double t = now_us();
    std::lock_guard<std::mutex> lk(mu);
    for (long id : sl.reqs) {
        auto it = reqs.find(id);
        if (it == reqs.end()) continue;
        it->second.done = true;
        it->second.t_done = t;
        lat_us.push_back(t - it->second.t_submit);
        ++completed;
        --inflight;
    }
    t_last = t;
    sl.reqs.clear();
    sl.busy = false;
    cv_done.notify_all();
}

bool spc5cuda_server::dispatch(Slot& sl) {
    int mat = -1;
    {
        std::lock_guard<std::mutex> lk(mu);
        double oldest = 0.0;
        for (auto& kv : pending) {
            if (kv.second.empty()) continue;
            const double t = reqs[kv.second.front()].t_submit;
            if (mat < 0 || t < oldest) {
                oldest = t;
                mat = kv.first;
            }
        }
        if (mat < 0) return false;
        auto& q = pending[mat];
        sl.reqs.clear();
        while (!q.empty() && int(sl.reqs.size()) < cfg.max_k) {
            sl.reqs.push_back(q.front());
            q.pop_front();
        }
    }
    const spc5cuda_mat* m = mats[size_t(mat)];
    const int k = int(sl.reqs.size());
    const size_t xb = cfg.mixed ? 4 : 8;
    const size_t yb = 8;
    const long ldX = max_cols, ldY = max_rows;
    std::vector<std::pair<const void*, void*>> io;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (long id : sl.reqs) io.emplace_back(reqs[id].x, reqs[id].y);
    }
    if (k == 1) {
        // a lone request: an SpMV straight into its own y, no staging copies
        void* y0 = io[0].second;
        SPC5_CUDA(cudaMemsetAsync(y0, 0, size_t(m->nrows) * yb, sl.stream));
        if (m->use_plan())
            plan_spmv(m, io[0].first, y0, cfg.mixed, sl.stream, cfg.plan_serial == 0);
        else if (cfg.mixed && m->value_type == SPC5CUDA_F32_V8)
            launch_spmv_mixed8(m->view(), static_cast<const float*>(io[0].first), static_cast<double*>(y0),
                               sl.stream);
        else if (cfg.mixed)
            launch_spmv_mixed(m->view(), static_cast<const float*>(io[0].first), static_cast<double*>(y0),
                              sl.stream);
        else
            launch_spmv_f64(m->view(), static_cast<const double*>(io[0].first), static_cast<double*>(y0),
                            sl.stream);
        return finish_dispatch(sl, k);
    }
    char* X = sl.X.as<char>();
    char* Y = sl.Y.as<char>();
    for (int q = 0; q < k; ++q)
        SPC5_CUDA(cudaMemcpyAsync(X + size_t(q) * ldX * xb, io[size_t(q)].first, size_t(m->ncols) * xb,
                                  cudaMemcpyDeviceToDevice, sl.stream));
    SPC5_CUDA(cudaMemsetAsync(Y, 0, size_t(k) * ldY * yb, sl.stream));
    if (m->use_plan())
        plan_spmm(m, k, X, 1, ldX, Y, 1, ldY, cfg.mixed, sl.stream, cfg.plan_serial == 0);
    else if (cfg.mixed && m->value_type == SPC5CUDA_F32_V8)
        launch_spmm_mixed8(m->spmm_view(), k, reinterpret_cast<const float*>(X), 1, ldX,
                           reinterpret_cast<double*>(Y), 1, ldY, sl.stream);
    else if (cfg.mixed)
        launch_spmm_mixed(m->spmm_view(), k, reinterpret_cast<const float*>(X), 1, ldX,
                          reinterpret_cast<double*>(Y), 1, ldY, sl.stream);
    else
        launch_spmm_f64(m->spmm_view(), k, reinterpret_cast<const double*>(X), 1, ldX,
                        reinterpret_cast<double*>(Y), 1, ldY, sl.stream);
    for (int q = 0; q < k; ++q)
        SPC5_CUDA(cudaMemcpyAsync(io[size_t(q)].second, Y + size_t(q) * ldY * yb, size_t(m->nrows) * yb,
                                  cudaMemcpyDeviceToDevice, sl.stream));
    return finish_dispatch(sl, k);
}

bool spc5cuda_server::finish_dispatch(Slot& sl, int k) {
    SPC5_CUDA(cudaEventRecord(sl.event, sl.stream));
    sl.busy = true;
    {
        std::lock_guard<std::mutex> lk(mu);
        ++launches;
        coalesced += k;
    }
    return true;
}

void spc5cuda_server::run() {
    try {
        SPC5_CUDA(cudaSetDevice(device));
        for (;;) {
            bool progress = false;
            for (auto& sl : slots) {
                if (sl.busy) {
                    const cudaError_t e = cudaEventQuery(sl.event);
                    if (e == cudaSuccess) {
                        complete(sl);
                        progress = true;
                    } else if (e != cudaErrorNotReady) {
                        check_cuda(e, "cudaEventQuery");
                    }
                }
            }
            for (auto& sl : slots) {
                if (!sl.busy && dispatch(sl)) progress = true;
            }
            std::unique_lock<std::mutex> lk(mu);
            if (stop) {
                bool any = false;
                for (auto& sl : slots) any = any || sl.busy;
                if (!any) break;
            }
            if (!progress) {
                bool busy = false;
                for (auto& sl : slots) busy = busy || sl.busy;
                bool queued = false;
                for (auto& kv : pending) queued = queued || !kv.second.empty();
                if (!busy && !queued && !stop) {
                    cv_work.wait_for(lk, std::chrono::milliseconds(5));
                } else {
                    lk.unlock();
                    std::this_thread::yield();
                }
            }
        }
    } catch (const Error& e) {
        std::lock_guard<std::mutex> lk(mu);
        error = e.status;
        stop = true;
        cv_done.notify_all();
    }
}

extern "C" {

spc5cuda_status spc5cuda_server_create(spc5cuda_server** out, const spc5cuda_server_config* cfg) {
    return guarded([&] {
        require(out && cfg, SPC5CUDA_ERR_INVALID, "null");
        require(cfg->slots >= 1 && cfg->slots <= 64 && cfg->max_k >= 1 && cfg->max_k <= 16 &&
                    cfg->hbm_budget > 0,
                SPC5CUDA_ERR_INVALID, "config");
        auto* sv = new spc5cuda_server();
        sv->cfg = *cfg;
        SPC5_CUDA(cudaGetDevice(&sv->device));
        sv->slots.resize(size_t(cfg->slots));
        for (auto& sl : sv->slots) {
            SPC5_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
            SPC5_CUDA(cudaEventCreateWithFlags(&sl.event, cudaEventDisableTiming));
        }
        sv->worker = std::thread([sv] { sv->run(); });
        *out = sv;
    });
}

spc5cuda_status spc5cuda_server_add_matrix(spc5cuda_server* sv, spc5cuda_mat* m, int* id) {
    return guarded([&] {
        require(sv && m && id, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "served matrices must be converted");
        require(sv->cfg.mixed ? (m->value_type == SPC5CUDA_F32 || m->value_type == SPC5CUDA_F32_V8)
                              : m->value_type == SPC5CUDA_F64,
                SPC5CUDA_ERR_FORMAT, "value type does not match the server");
        std::unique_lock<std::mutex> lk(sv->mu);
        require(sv->inflight == 0, SPC5CUDA_ERR_INVALID, "add matrices while the server is idle");
        const int rows = std::max(sv->max_rows, m->nrows);
        const int cols = std::max(sv->max_cols, m->ncols);
        const long need = sv->resident_bytes + m->device_bytes() + sv->slot_bytes(rows, cols);
        require(need <= sv->cfg.hbm_budget, SPC5CUDA_ERR_NOMEM, "HBM budget exceeded");
        if (rows != sv->max_rows || cols != sv->max_cols) {
            const size_t xb = sv->cfg.mixed ? 4 : 8;
            for (auto& sl : sv->slots) {
                sl.X.alloc(size_t(cols) * size_t(sv->cfg.max_k) * xb);
                sl.Y.alloc(size_t(rows) * size_t(sv->cfg.max_k) * 8);
            }
            sv->max_rows = rows;
            sv->max_cols = cols;
        }
        sv->resident_bytes += m->device_bytes();
        sv->mats.push_back(m);
        *id = int(sv->mats.size()) - 1;
    });
}

spc5cuda_status spc5cuda_server_submit(spc5cuda_server* sv, int id, const void* x, void* y,
                                       long* req_id) {
    return guarded([&] {
        require(sv && x && y && req_id, SPC5CUDA_ERR_INVALID, "null");
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->error != SPC5CUDA_OK) throw Error(sv->error, "server failed");
        require(id >= 0 && id < int(sv->mats.size()), SPC5CUDA_ERR_INVALID, "matrix id");
        const long rid = sv->next_id++;
        Request r;
        r.mat = id;
        r.x = x;
        r.y = y;
        r.t_submit = now_us();
        if (sv->t_first == 0.0) sv->t_first = r.t_submit;
        sv->reqs.emplace(rid, r);
        sv->pending[id].push_back(rid);
        ++sv->inflight;
        *req_id = rid;
        sv->cv_work.notify_one();
    });
}

spc5cuda_status spc5cuda_server_wait(spc5cuda_server* sv, long req_id, double timeout_s,
                                     double* latency_us) {
    return guarded([&] {
        require(sv != nullptr, SPC5CUDA_ERR_INVALID, "null");
        std::unique_lock<std::mutex> lk(sv->mu);
        auto it = sv->reqs.find(req_id);
        require(it != sv->reqs.end(), SPC5CUDA_ERR_INVALID, "unknown request");
        const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s);
        while (!it->second.done && sv->error == SPC5CUDA_OK) {
            if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !it->second.done)
                throw Error(SPC5CUDA_ERR_TIMEOUT, "request not finished");
        }
        if (sv->error != SPC5CUDA_OK) throw Error(sv->error, "server failed");
        if (latency_us) *latency_us = it->second.t_done - it->second.t_submit;
        sv->reqs.erase(it);
    });
}

spc5cuda_status spc5cuda_server_drain(spc5cuda_server* sv, double timeout_s) {
    return guarded([&] {
        require(sv != nullptr, SPC5CUDA_ERR_INVALID, "null");
        std::unique_lock<std::mutex> lk(sv->mu);
        const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s);
        while (sv->inflight > 0 && sv->error == SPC5CUDA_OK) {
            if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && sv->inflight > 0)
                throw Error(SPC5CUDA_ERR_TIMEOUT, "requests still in flight");
        }
        if (sv->error != SPC5CUDA_OK) throw Error(sv->error, "server failed");
        for (auto it = sv->reqs.begin(); it != sv->reqs.end();) {
            if (it->second.done) it = sv->reqs.erase(it);
            else ++it;
        }
    });
}

spc5cuda_status spc5cuda_server_get_stats(spc5cuda_server* sv, spc5cuda_server_stats* st, int reset) {
    return guarded([&] {
        require(sv && st, SPC5CUDA_ERR_INVALID, "null");
        std::lock_guard<std::mutex> lk(sv->mu);
        std::vector<double> l = sv->lat_us;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            if (l.empty()) return 0.0;
            const size_t i = std::min(l.size() - 1, size_t(p * double(l.size() - 1) + 0.5));
            return l[i];
        };
        st->completed = sv->completed;
        st->launches = sv->launches;
        st->mean_k = sv->launches ? double(sv->coalesced) / double(sv->launches) : 0.0;
        st->p50_us = pct(0.50);
        st->p99_us = pct(0.99);
        st->max_us = l.empty() ? 0.0 : l.back();
        const double span = sv->t_last - sv->t_first;
        st->req_per_s = span > 0 ? double(sv->completed) / (span * 1e-6) : 0.0;
        st->resident_bytes = sv->resident_bytes;
        st->matrices = int(sv->mats.size());
        if (reset) {
            sv->lat_us.clear();
            sv->completed = 0;
            sv->launches = 0;
            sv->coalesced = 0;
            sv->t_first = sv->t_last = 0.0;
        }
    });
}

spc5cuda_status spc5cuda_server_destroy(spc5cuda_server* sv) {
    return guarded([&] {
        if (!sv) return;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->stop = true;
            sv->cv_work.notify_all();
        }
        if (sv->worker.joinable()) sv->worker.join();
        for (auto& sl : sv->slots) {
            if (sl.event) cudaEventDestroy(sl.event);
            if (sl.stream) cudaStreamDestroy(sl.stream);
        }
        delete sv;
    });
}

}  // extern "C"
