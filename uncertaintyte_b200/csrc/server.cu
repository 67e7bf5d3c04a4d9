// server.cu - a request loop for many reconstructions on one GPU (host code).
//
// The reference computes one reconstruction per call and is not re-entrant
// (global MAGMA init/finalize and a fixed OpenMP thread count per call,
// compute.cpp:461-468, 539). This server has no counterpart there: callers
// submit reconstructions of any size as they arrive and wait for them later.
//
// * Continuous batching: `max_inflight` worker threads, each with its own
//   context (CUDA stream + device workspace kept between requests). A request
//   that arrives while others run starts as soon as a worker is free and its
//   device memory fits; the kernels of all running requests overlap on the GPU
//   (different streams), the host-side waits of one request block only its
//   worker.
// * Admission by device-memory footprint (unc_request_bytes: the dense Schur
//   complement and its inverse buffers, the block storage, the int8
//   slices): the sum over running requests and idle workspaces stays
//   within `max_device_bytes`. A worker holds two workspaces (its context's,
//   grown by single requests, and its batch's, grown by packs), and both are
//   counted: a run grows one of them while the other keeps its memory, unless
//   the worker frees it first to make room. Idle workers' workspaces are
//   released when that makes a request fit. Later requests may start ahead
//   of a waiting one (backfill) at most kMaxBypass times, so large requests
//   are not starved.
// * Small requests (footprint <= kSmallBytes) run on high-priority streams,
//   so the block scheduler serves their kernels ahead of a large request's
//   GEMM tiles, and a quarter of the workers take small requests only, so a
//   burst of large requests cannot hold every slot.
// * Packing: a worker that starts a small request also takes the other small
//   requests waiting behind it (up to kMaxPack, within the memory budget) and
//   runs them as one grouped batch (unc_batch_compute: one launch sequence,
//   replayed from a CUDA graph when the pack's shape repeats).
// * Each result depends only on its own inputs (no atomics in the arithmetic,
//   fixed reduction orders): alone or in a mix, a request gives the same bytes.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/uncte.h"
#include "admission.h"
#include "internal.h"

namespace {

constexpr long long kSmallBytes = 1LL << 30;

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    unc_options opt{};
    int num_rows = 0, num_cols = 0;
    const int* rows = nullptr;
    const int* cols = nullptr;
    const double* vals = nullptr;
    double* cam = nullptr;
    double* pt = nullptr;
    long long bytes = 0;
    bool small = false;
    int bypassed = 0;
    bool done = false;
    bool waited = false;  // a thread is inside unc_server_wait for this request
    int status = UNC_OK;
    std::string error;
    unc_statistic st{};
    Clock::time_point t_submit, t_start, t_end;
};

struct Worker {
    unc_context* ctx = nullptr;
    unc_batch* batch = nullptr;  // packs of small requests
    long long committed = 0;  // device bytes held or promised (workspace, or the running request's footprint)
    // What the two workspaces hold between runs: a single request grows the
    // context's, a pack the batch's, and each keeps its memory after the run.
    long long ctx_held = 0, batch_held = 0;
    bool drop_ctx = false, drop_batch = false;  // free that workspace before the next run (room for it)
    bool busy = false;
    bool releasing = false;   // another worker is freeing this one's workspaces
    bool small_only = false;  // reserved for small requests
    std::thread th;
};

}  // namespace

struct unc_server {
    int device = 0;
    long long budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::unordered_map<long long, std::shared_ptr<Request>> all;
    std::vector<std::unique_ptr<Worker>> workers;
    long long next_id = 1;
    bool stopping = false;
    int running = 0;
    long long completed = 0;
};

namespace {

void worker_loop(unc_server* s, Worker* w) {
    cudaSetDevice(s->device);
    if (unc_context_create(s->device, &w->ctx) != UNC_OK) w->ctx = nullptr;
    // requests run side by side: each tile-task inverse takes about two workers' share of the SMs
    const int sms = unc::device_sms();
    if (w->ctx) unc::context_set_task_ctas(w->ctx, (2 * sms + (int)s->workers.size() - 1) / (int)s->workers.size());
    std::unique_lock<std::mutex> lk(s->mu);
    std::vector<Worker*> release;
    for (;;) {
        std::vector<std::shared_ptr<Request>> pack;
        s->cv_work.wait(lk, [&] {
            return !(pack = unc_admission::pick(s, w, release)).empty() ||
                   (s->stopping && s->pending.empty() && !w->releasing);
        });
        if (pack.empty()) break;
        w->busy = true;
        s->running += (int)pack.size();
        lk.unlock();
        if (!release.empty()) {
            // the idle workers picked for release wait (releasing) until this is done
            for (Worker* v : release) {
                if (v->ctx) unc_context_release(v->ctx);
                if (v->batch) unc_batch_release(v->batch);
            }
            lk.lock();
            for (Worker* v : release) v->releasing = false;
            s->cv_work.notify_all();
            lk.unlock();
        }
        // this worker's own other workspace, when the admission counted it as freed
        if (w->drop_ctx && w->ctx) unc_context_release(w->ctx);
        if (w->drop_batch && w->batch) unc_batch_release(w->batch);
        const auto t_start = Clock::now();
        for (auto& r : pack) r->t_start = t_start;
        std::vector<int> rcs(pack.size(), UNC_ERR_CUDA);
        std::vector<std::string> errs(pack.size());
        if (pack.size() == 1) {
            auto& r = pack[0];
            if (w->ctx) unc_context_set_priority(w->ctx, r->small ? 1 : 0);
            rcs[0] = w->ctx ? unc_compute(w->ctx, &r->opt, r->num_rows, r->num_cols, r->rows, r->cols, r->vals,
                                          r->cam, r->pt, &r->st)
                            : UNC_ERR_CUDA;
            if (rcs[0] != UNC_OK) errs[0] = unc_last_error();
        } else {
            if (!w->batch && unc_batch_create(s->device, &w->batch) != UNC_OK) w->batch = nullptr;
            const size_t n = pack.size();
            std::vector<unc_options> opts(n);
            std::vector<int> nr(n), nc(n);
            std::vector<const int*> rows(n), cols(n);
            std::vector<const double*> vals(n);
            std::vector<double*> cam(n), pt(n);
            std::vector<unc_statistic> st(n);
            for (size_t k = 0; k < n; ++k) {
                opts[k] = pack[k]->opt;
                nr[k] = pack[k]->num_rows;
                nc[k] = pack[k]->num_cols;
                rows[k] = pack[k]->rows;
                cols[k] = pack[k]->cols;
                vals[k] = pack[k]->vals;
                cam[k] = pack[k]->cam;
                pt[k] = pack[k]->pt;
            }
            int rc = w->batch ? unc_batch_compute(w->batch, (int)n, opts.data(), nr.data(), nc.data(), rows.data(),
                                                  cols.data(), vals.data(), cam.data(), pt.data(), rcs.data(), st.data())
                              : UNC_ERR_CUDA;
            const std::string msg = unc_last_error();
            for (size_t k = 0; k < n; ++k) {
                if (rc != UNC_OK) rcs[k] = rc;
                if (rcs[k] != UNC_OK) errs[k] = rc != UNC_OK ? msg : std::string(unc_status_string(rcs[k]));
                pack[k]->st = st[k];
            }
        }
        const auto t_end = Clock::now();
        lk.lock();
        for (size_t k = 0; k < pack.size(); ++k) {
            pack[k]->t_end = t_end;
            pack[k]->status = rcs[k];
            pack[k]->error = errs[k];
            pack[k]->done = true;
        }
        w->busy = false;
        unc_admission::settle(w, w->ctx ? unc_context_device_bytes(w->ctx) : 0,
                              w->batch ? unc_batch_device_bytes(w->batch) : 0);
        s->running -= (int)pack.size();
        s->completed += (long long)pack.size();
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // memory may have come free for a waiting request
    }
    lk.unlock();
    if (w->batch) unc_batch_destroy(w->batch);
    w->batch = nullptr;
    if (w->ctx) unc_context_destroy(w->ctx);
    w->ctx = nullptr;
}

}  // namespace

extern "C" {

int unc_server_create(int device, long long max_device_bytes, int max_inflight, unc_server** out) {
    if (!out || max_inflight <= 0 || max_inflight > 64) {
        unc::g_last_error = "unc_server_create: out must be non-NULL and max_inflight in 1..64";
        return UNC_ERR_INVALID_ARG;
    }
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
        unc::g_last_error = std::string("unc_server_create: ") + cudaGetErrorString(e);
        return UNC_ERR_CUDA;
    }
    auto* s = new unc_server();
    s->device = device;
    s->budget = max_device_bytes > 0 ? max_device_bytes : (long long)(free_b / 10 * 9);
    for (int i = 0; i < max_inflight; ++i) s->workers.emplace_back(new Worker());
    for (int i = 0; i < max_inflight / 4; ++i) s->workers[i]->small_only = true;
    for (auto& w : s->workers) w->th = std::thread(worker_loop, s, w.get());
    *out = s;
    return UNC_OK;
}

int unc_server_submit(unc_server* s, const unc_options* opt, int num_rows, int num_cols, const int* rows,
                      const int* cols, const double* values, double* cam_unc, double* pt_unc, long long* id) {
    if (!s || !opt || !rows || !cols || !values || !cam_unc || !pt_unc || !id) {
        unc::g_last_error = "unc_server_submit: null argument";
        return UNC_ERR_INVALID_ARG;
    }
    const long long bytes = unc_request_bytes(opt, num_rows, num_cols, rows, cols);
    if (bytes < 0) return unc_compute(nullptr, opt, num_rows, num_cols, rows, cols, values, cam_unc, pt_unc,
                                      nullptr);  // reports the option error without running anything
    auto r = std::make_shared<Request>();
    r->opt = *opt;
    r->num_rows = num_rows;
    r->num_cols = num_cols;
    r->rows = rows;
    r->cols = cols;
    r->vals = values;
    r->cam = cam_unc;
    r->pt = pt_unc;
    r->bytes = bytes;
    r->small = bytes <= kSmallBytes;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) {
        unc::g_last_error = "unc_server_submit: server is shutting down";
        return UNC_ERR_INVALID_ARG;
    }
    if (bytes > s->budget) {
        unc::g_last_error = "unc_server_submit: request needs " + std::to_string(bytes) +
                            " device bytes, above the server's budget of " + std::to_string(s->budget);
        return UNC_ERR_OUT_OF_MEMORY;
    }
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->pending.push_back(r);
    *id = r->id;
    s->cv_work.notify_all();
    return UNC_OK;
}

int unc_server_wait(unc_server* s, long long id, double timeout_s, int* status, unc_statistic* st,
                    double* latency_s, double* queue_s) {
    if (!s) {
        unc::g_last_error = "unc_server_wait: server is NULL";
        return UNC_ERR_INVALID_ARG;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) {
        unc::g_last_error = "unc_server_wait: unknown request id (or already collected)";
        return UNC_ERR_INVALID_ARG;
    }
    // Only the shared_ptr is kept across the wait: submits from other threads
    // insert into `all` meanwhile, and a rehash invalidates every iterator.
    std::shared_ptr<Request> r = it->second;
    if (r->waited) {
        unc::g_last_error = "unc_server_wait: another thread is already waiting for this request";
        return UNC_ERR_INVALID_ARG;
    }
    r->waited = true;
    auto ready = [&] { return r->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        r->waited = false;
        unc::g_last_error = "unc_server_wait: request still running";
        return UNC_ERR_TIMEOUT;
    }
    s->all.erase(id);
    if (status) *status = r->status;
    if (st) *st = r->st;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_end - r->t_submit).count();
    if (queue_s) *queue_s = std::chrono::duration<double>(r->t_start - r->t_submit).count();
    if (r->status != UNC_OK) unc::g_last_error = r->error;
    return UNC_OK;
}

int unc_server_destroy(unc_server* s) {
    if (!s) return UNC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_work.notify_all();
    }
    for (auto& w : s->workers)
        if (w->th.joinable()) w->th.join();
    delete s;
    return UNC_OK;
}

}  // extern "C"
