// spj_server.cu -- the served join stream: continuous batching on one GPU.
//
// Clients submit joins over device-resident columns. A worker thread admits
// queued requests in arrival order while their HBM footprint (columns, output
// and partition scratch) fits the server's budget, turns everything admitted at
// that moment into ONE batch plan (the spj_batch_* pipeline: one launch
// sequence, per-join tuning, one unit queue) and launches it on a free stream,
// so a batch formed while others still run overlaps with them on the device.
// Scratch comes from a private stream-ordered memory pool (cudaMallocAsync
// semantics, memory kept reserved between batches), so admitting a batch never
// synchronises the device. A batch retires when its event completes; a
// request's latency runs from its submit call to that moment.
//
// There is no counterpart in the reference, which runs one JoinInstance per
// join, one join at a time.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "spj_internal.h"

using namespace spj;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    const spj_kv_pair_t *r = nullptr, *s = nullptr;
    int64_t n_r = 0, n_s = 0;
    spj_kv_pair_t *out = nullptr;
    int64_t *n_out = nullptr;
    uint64_t resident = 0;  // columns + output, held until the request completes
    uint64_t estimate = 0;  // resident + expected partition scratch
    Clock::time_point t_submit, t_done;
    int status = 1;  // 1 = queued or running, 0 = done, < 0 = SPJ_E_* code
    std::string message;
};

// One stream and what is running on it.
struct Flight {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    JoinCtr *host_ctr = nullptr;  // pinned, max_batch entries: the batch's counters
    spj_plan_t *plan = nullptr;   // null when the stream is free
    std::vector<Request *> reqs;
    uint64_t bytes = 0;  // accounted against the budget while in flight
};

// Expected partition scratch of one join in a batch plan: the two partition
// passes each hold a copy of both relations.
uint64_t scratch_estimate(int64_t n_r, int64_t n_s) { return 16ull * (uint64_t)(n_r + n_s) + (1ull << 20); }

}  // namespace

struct spj_server {
    spj_design_t design{};
    uint64_t budget = 0, used = 0, peak = 0;
    int max_batch = 64;
    int device = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<Flight> flights;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<int64_t, Request *> reqs;
    int64_t next_id = 0, submitted = 0, completed = 0, failed = 0, batches = 0, batched_reqs = 0;
    int max_inflight = 0;
    std::vector<double> latencies_ms;
    bool stop = false;
    bool held = false;  // admission paused by spj_server_hold
    std::thread worker;
};

// Called with the lock held; makes no CUDA call that can wait on the device.
static void retire(spj_server *sv, Flight &f) {
    const auto now = Clock::now();
    for (size_t j = 0; j < f.reqs.size(); j++) {
        Request *q = f.reqs[j];
        q->t_done = now;
        q->status = join_ctr_status(f.host_ctr[j].error, f.host_ctr[j].max_r_part);
        if (q->status != SPJ_OK) {
            q->message = spj_last_error();
            sv->failed++;
        }
        sv->latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - q->t_submit).count());
    }
    destroy_plan_stream(f.plan, f.stream);
    sv->used -= f.bytes;
    sv->completed += (int64_t)f.reqs.size();
    f.plan = nullptr;
    f.reqs.clear();
    f.bytes = 0;
}

static void fail_batch(spj_server *sv, std::vector<Request *> &take, int rc, const std::string &msg) {
    const auto now = Clock::now();
    for (auto *q : take) {
        q->status = rc;
        q->message = msg;
        q->t_done = now;
    }
    sv->completed += (int64_t)take.size();
    sv->failed += (int64_t)take.size();
}

static void worker_loop(spj_server *sv) {
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        bool retired = false;
        int inflight = 0, slot = -1;
        for (size_t i = 0; i < sv->flights.size(); i++) {
            Flight &f = sv->flights[i];
            if (f.plan && cudaEventQuery(f.done) == cudaSuccess) {
                retire(sv, f);
                retired = true;
            }
            if (f.plan)
                inflight++;
            else if (slot < 0)
                slot = (int)i;
        }
        if (retired) sv->cv_done.notify_all();
        if (sv->stop && sv->queue.empty() && inflight == 0) break;

        // Admit, in arrival order, what fits the budget. A request larger than
        // the whole budget runs alone once nothing else is in flight.
        std::vector<Request *> take;
        uint64_t est = 0;
        if (slot >= 0 && (!sv->held || sv->stop)) {
            while (!sv->queue.empty() && (int)take.size() < sv->max_batch) {
                Request *q = sv->queue.front();
                const bool alone = take.empty() && inflight == 0;
                if (sv->used + est + q->estimate > sv->budget && !alone) break;
                take.push_back(q);
                est += q->estimate;
                sv->queue.pop_front();
            }
        }
        if (take.empty()) {
            sv->cv_work.wait_for(lk, std::chrono::microseconds(inflight ? 20 : 2000));
            continue;
        }
        Flight &f = sv->flights[slot];
        sv->used += est;  // provisional, replaced by the exact figure below
        sv->peak = std::max(sv->peak, sv->used);
        lk.unlock();

        const int J = (int)take.size();
        std::vector<int64_t> nr(J), ns(J);
        std::vector<const spj_kv_pair_t *> r(J), s(J);
        std::vector<spj_kv_pair_t *> o(J);
        std::vector<int64_t *> cnt(J);
        uint64_t resident = 0;
        for (int j = 0; j < J; j++) {
            nr[j] = take[j]->n_r;
            ns[j] = take[j]->n_s;
            r[j] = take[j]->r;
            s[j] = take[j]->s;
            o[j] = take[j]->out;
            cnt[j] = take[j]->n_out;
            resident += take[j]->resident;
        }
        spj_plan_t *pl = nullptr;
        size_t scratch = 0;
        int rc = create_plan_stream(J, nr.data(), ns.data(), &sv->design, r.data(), s.data(), o.data(), cnt.data(),
                                    sv->pool, f.stream, &pl, &scratch);
        if (rc == SPJ_OK) rc = spj_batch_execute(pl, f.stream);
        if (rc == SPJ_OK) {
            cudaError_t e = cudaMemcpyAsync(f.host_ctr, pl->dev.jctr, J * sizeof(JoinCtr), cudaMemcpyDeviceToHost,
                                            f.stream);
            if (e == cudaSuccess) e = cudaEventRecord(f.done, f.stream);
            if (e != cudaSuccess) rc = cuda_error(e, "batch completion record");
        }
        const std::string msg = rc == SPJ_OK ? std::string() : std::string(spj_last_error());
        if (rc != SPJ_OK && pl) {
            cudaStreamSynchronize(f.stream);  // the lock is not held here
            destroy_plan_stream(pl, f.stream);
            pl = nullptr;
        }

        lk.lock();
        sv->used -= est;
        if (rc != SPJ_OK) {
            fail_batch(sv, take, rc, msg);
            sv->cv_done.notify_all();
            continue;
        }
        f.plan = pl;
        f.reqs = std::move(take);
        f.bytes = resident + scratch;
        sv->used += f.bytes;
        sv->peak = std::max(sv->peak, sv->used);
        sv->batches++;
        sv->batched_reqs += J;
        sv->max_inflight = std::max(sv->max_inflight, inflight + 1);
    }
}

extern "C" {

int spj_server_create(const spj_design_t *design, uint64_t hbm_budget_bytes, int max_batch, int streams,
                      spj_server_t **out) {
    if (!out || !design) return set_error(SPJ_E_ARG, "NULL argument");
    *out = nullptr;
    if (max_batch < 1 || max_batch > 4096 || streams < 1 || streams > 64 || hbm_budget_bytes == 0)
        return set_error(SPJ_E_ARG, "server limits: 1 <= max_batch <= 4096, 1 <= streams <= 64, budget > 0");
    if (design->join_alg < 0 || design->join_alg > 3) return set_error(SPJ_E_ARG, "bad join_alg");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    spj_server *sv = new spj_server();
    sv->design = *design;
    sv->budget = hbm_budget_bytes;
    sv->max_batch = max_batch;
    cudaGetDevice(&sv->device);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = sv->device;
    cudaError_t e = cudaMemPoolCreate(&sv->pool, &props);
    if (e == cudaSuccess) {
        uint64_t keep = hbm_budget_bytes;  // keep freed scratch reserved for the next batches
        e = cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    sv->flights.resize(streams);
    for (int i = 0; i < streams && e == cudaSuccess; i++) {
        Flight &f = sv->flights[i];
        e = cudaStreamCreateWithFlags(&f.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost(&f.host_ctr, (size_t)max_batch * sizeof(JoinCtr));
    }
    if (e != cudaSuccess) {
        const int rc = cuda_error(e, "server set-up");
        spj_server_destroy(sv);
        return rc;
    }
    sv->worker = std::thread(worker_loop, sv);
    *out = sv;
    return SPJ_OK;
}

int64_t spj_server_output_capacity(spj_server_t *sv, int64_t n_r, int64_t n_s) {
    if (!sv || n_r < 0 || n_s < 0) {
        set_error(SPJ_E_ARG, "bad argument");
        return -1;
    }
    return join_output_capacity(n_r, n_s, sv->design, false);
}

int spj_server_submit(spj_server_t *sv, const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s, int64_t n_s,
                      spj_kv_pair_t *out, int64_t out_capacity, int64_t *n_out, int64_t *id) {
    if (!sv || !out || !n_out || !id) return set_error(SPJ_E_ARG, "NULL argument");
    if (n_r < 0 || n_s < 0 || n_r >= kMaxTuples || n_s >= kMaxTuples || (n_r && !r) || (n_s && !s))
        return set_error(SPJ_E_ARG, "bad columns");
    if (((uintptr_t)r & 15) || ((uintptr_t)s & 15) || ((uintptr_t)out & 15) || ((uintptr_t)n_out & 7))
        return set_error(SPJ_E_ARG, "columns and output must be 16-byte aligned, the count 8-byte aligned");
    const int64_t need = spj_server_output_capacity(sv, n_r, n_s);
    if (need < 0) return SPJ_E_ARG;
    if (out_capacity < need) return set_error(SPJ_E_ARG, "out_capacity below spj_server_output_capacity()");
    Request *q = new Request();
    q->r = r;
    q->s = s;
    q->n_r = n_r;
    q->n_s = n_s;
    q->out = out;
    q->n_out = n_out;
    q->resident = 8ull * (uint64_t)(n_r + n_s) + 8ull * (uint64_t)out_capacity;
    q->estimate = q->resident + scratch_estimate(n_r, n_s);
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) {
            delete q;
            return set_error(SPJ_E_STATE, "server is shutting down");
        }
        q->id = sv->next_id++;
        sv->reqs[q->id] = q;
        sv->queue.push_back(q);
        sv->submitted++;
        *id = q->id;
    }
    sv->cv_work.notify_one();
    return SPJ_OK;
}

int spj_server_wait(spj_server_t *sv, int64_t id, double timeout_ms, double *latency_ms) {
    if (!sv) return set_error(SPJ_E_ARG, "server is NULL");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return set_error(SPJ_E_ARG, "unknown or already collected request id");
    Request *q = it->second;
    auto finished = [q] { return q->status != 1; };
    if (timeout_ms < 0)
        sv->cv_done.wait(lk, finished);
    else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), finished))
        return set_error(SPJ_E_TIMEOUT, "request still running");
    const int st = q->status;
    const std::string msg = q->message;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
    sv->reqs.erase(it);
    delete q;
    lk.unlock();
    return st == SPJ_OK ? SPJ_OK : set_error(st, msg.empty() ? "join failed" : msg);
}

int spj_server_stats(spj_server_t *sv, spj_server_stats_t *out) {
    if (!sv || !out) return set_error(SPJ_E_ARG, "NULL argument");
    std::vector<double> l;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        memset(out, 0, sizeof(*out));
        out->submitted = sv->submitted;
        out->completed = sv->completed;
        out->failed = sv->failed;
        out->batches = sv->batches;
        out->max_inflight_batches = sv->max_inflight;
        out->mean_batch = sv->batches ? (double)sv->batched_reqs / (double)sv->batches : 0.0;
        out->hbm_peak_bytes = sv->peak;
        out->hbm_budget_bytes = sv->budget;
        l = sv->latencies_ms;
    }
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        out->p50_ms = l[(l.size() - 1) / 2];
        out->p99_ms = l[(size_t)((double)(l.size() - 1) * 0.99)];
        out->max_ms = l.back();
    }
    return SPJ_OK;
}

int spj_server_hold(spj_server_t *sv, int hold) {
    if (!sv) return set_error(SPJ_E_ARG, "server is NULL");
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->held = hold != 0;
    }
    sv->cv_work.notify_all();
    return SPJ_OK;
}

int spj_server_reset_stats(spj_server_t *sv) {
    if (!sv) return set_error(SPJ_E_ARG, "server is NULL");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->latencies_ms.clear();
    sv->submitted = (int64_t)sv->queue.size();
    for (auto &f : sv->flights) sv->submitted += (int64_t)f.reqs.size();
    sv->completed = sv->failed = sv->batches = sv->batched_reqs = 0;
    sv->max_inflight = 0;
    sv->peak = sv->used;
    return SPJ_OK;
}

void spj_server_destroy(spj_server_t *sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();  // drains the queue and every batch in flight
    for (auto &f : sv->flights) {
        if (f.stream) cudaStreamSynchronize(f.stream);
        if (f.plan) retire(sv, f);
        if (f.done) cudaEventDestroy(f.done);
        if (f.host_ctr) cudaFreeHost(f.host_ctr);
        if (f.stream) cudaStreamDestroy(f.stream);
    }
    for (auto &kv : sv->reqs) delete kv.second;
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    delete sv;
}

}  // extern "C"
