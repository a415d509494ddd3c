// spj_instance.cu -- the JoinInstance-shaped handle of the C ABI
// (pidjoin::JoinInstance, include/join_internals.hpp:301-323 of yonsei-hpcp/spid-join).
//
// Reference flow: LoadColumn splits and aliases the caller's columns,
// PrepareJoin allocates ranks and spawns one thread per rank, StartJoin signals
// them, FinishJoin joins the threads and returns per-rank result buffers
// (src/query.cc:178-317, 1517-1567). Here: load_column borrows the column,
// prepare builds the device plan and its buffers, start enqueues the column
// copies and the join on the instance's stream, finish waits and copies the
// pairs back. One stream per instance; instances are independent.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "spj_internal.h"

using namespace spj;

struct spj_handle {
    int ranks = 1, rank_groups = 1, ranks_per_group = 1;
    const void *col[2] = {nullptr, nullptr};
    int64_t n[2] = {0, 0};
    bool col_set[2] = {false, false};
    bool on_device[2] = {false, false};
    spj_design_t design{};
    spj_plan_t *plan = nullptr;
    bool started = false;
    cudaStream_t stream = nullptr;
    spj_kv_pair_t *d_col[2] = {nullptr, nullptr};  // device copies of host columns
    int64_t d_cap[2] = {0, 0};
    spj_kv_pair_t *d_out = nullptr;
    int64_t d_out_cap = 0;
    int64_t *d_n = nullptr;
    int64_t *h_n = nullptr;           // pinned
    spj_kv_pair_t *h_out = nullptr;   // pinned
    int64_t h_out_cap = 0;
    int64_t n_pairs = 0;
    std::vector<int64_t> rank_off;
    cudaEvent_t ev[4]{};              // start, after h2d, after join, after d2h
    bool events = false;
    double d2h_ms = 0, h2d_ms = 0;
};

static int free_buffers(spj_handle_t *h) {
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_col[i]);
        h->d_col[i] = nullptr;
        h->d_cap[i] = 0;
    }
    cudaFree(h->d_out);
    h->d_out = nullptr;
    h->d_out_cap = 0;
    if (h->plan) spj_plan_destroy(h->plan);
    h->plan = nullptr;
    return SPJ_OK;
}

extern "C" {

int spj_create(int num_rank_allocated, int num_rankgroup, int num_rank_in_rankgroup, spj_handle_t **out) {
    if (!out) return set_error(SPJ_E_ARG, "out is NULL");
    *out = nullptr;
    if (num_rank_allocated < 1 || num_rankgroup < 1 || num_rank_in_rankgroup < 1 ||
        num_rankgroup * num_rank_in_rankgroup != num_rank_allocated)
        return set_error(SPJ_E_ARG, "ranks must equal rank groups x ranks per group");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    spj_handle_t *h = new spj_handle_t();
    h->ranks = num_rank_allocated;
    h->rank_groups = num_rankgroup;
    h->ranks_per_group = num_rank_in_rankgroup;
    spj_design_default(&h->design);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_n, sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_n, sizeof(int64_t));
    if (e != cudaSuccess) {
        spj_destroy(h);
        return cuda_error(e, "spj_create");
    }
    h->events = true;
    for (auto &ev : h->ev)
        if (cudaEventCreate(&ev) != cudaSuccess) h->events = false;
    *out = h;
    return SPJ_OK;
}

int spj_load_column(spj_handle_t *h, const void *tuples, int64_t num_tuples, int side) {
    if (!h) return set_error(SPJ_E_ARG, "handle is NULL");
    if (side != 0 && side != 1)
        return set_error(SPJ_E_ARG, "column must be \"left\" (0) or \"right\" (1)");  // src/query.cc:215-227
    if (num_tuples < 0 || (num_tuples > 0 && !tuples)) return set_error(SPJ_E_ARG, "bad column");
    if (h->started) return set_error(SPJ_E_STATE, "join in flight; call spj_finish first");
    cudaPointerAttributes attr;
    bool dev = false;
    if (tuples && cudaPointerGetAttributes(&attr, tuples) == cudaSuccess)
        dev = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    cudaGetLastError();
    h->col[side] = tuples;
    h->n[side] = num_tuples;
    h->on_device[side] = dev;
    h->col_set[side] = true;
    return SPJ_OK;
}

int spj_prepare(spj_handle_t *h, const spj_design_t *design) {
    if (!h) return set_error(SPJ_E_ARG, "handle is NULL");
    if (h->started) return set_error(SPJ_E_STATE, "join in flight; call spj_finish first");
    if (!h->col_set[0] || !h->col_set[1]) return set_error(SPJ_E_STATE, "load both columns before prepare");
    spj_design_t d = design ? *design : h->design;
    // the instance's rank layout is authoritative (JoinInstance(r, R, r/R))
    d.rank_num = h->ranks;
    d.rank_set = h->rank_groups;
    if (h->plan && h->plan->n_r == h->n[0] && h->plan->n_s == h->n[1] &&
        memcmp(&h->plan->design, &d, sizeof(d)) == 0) {
        h->design = d;
        return SPJ_OK;  // reuse the plan and its buffers
    }
    free_buffers(h);
    int rc = spj_plan_create(h->n[0], h->n[1], &d, &h->plan);
    if (rc) return rc;
    h->design = d;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; i++)
        if (!h->on_device[i] && h->n[i] > 0) {
            e = cudaMalloc(&h->d_col[i], (size_t)h->n[i] * 8);
            h->d_cap[i] = h->n[i];
        }
    h->d_out_cap = spj_plan_output_capacity(h->plan);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_out, (size_t)h->d_out_cap * 8);
    if (e == cudaSuccess && h->h_out_cap < h->n[1]) {
        cudaFreeHost(h->h_out);
        h->h_out = nullptr;
        h->h_out_cap = 0;
        e = cudaMallocHost(&h->h_out, (size_t)std::max<int64_t>(h->n[1], 1) * 8);
        if (e == cudaSuccess) h->h_out_cap = std::max<int64_t>(h->n[1], 1);
    }
    if (e != cudaSuccess) {
        free_buffers(h);
        return cuda_error(e, "spj_prepare buffers");
    }
    return SPJ_OK;
}

int spj_start(spj_handle_t *h, const spj_design_t *design) {
    if (!h) return set_error(SPJ_E_ARG, "handle is NULL");
    if (!h->plan) return set_error(SPJ_E_STATE, "spj_prepare must precede spj_start");
    if (h->started) return set_error(SPJ_E_STATE, "join already started");
    if (design) {
        spj_design_t d = *design;
        d.rank_num = h->ranks;
        d.rank_set = h->rank_groups;
        if (memcmp(&d, &h->design, sizeof(d)) != 0) {
            int rc = spj_prepare(h, &d);
            if (rc) return rc;
        }
    }
    if (h->events) cudaEventRecord(h->ev[0], h->stream);
    const spj_kv_pair_t *col[2];
    for (int i = 0; i < 2; i++) {
        if (h->n[i] == 0) {
            col[i] = h->d_out;  // never read; any aligned device pointer
        } else if (h->on_device[i]) {
            col[i] = (const spj_kv_pair_t *)h->col[i];
        } else {
            cudaError_t e = cudaMemcpyAsync(h->d_col[i], h->col[i], (size_t)h->n[i] * 8, cudaMemcpyHostToDevice,
                                            h->stream);
            if (e != cudaSuccess) return cuda_error(e, "column copy");
            col[i] = h->d_col[i];
        }
    }
    if (h->events) cudaEventRecord(h->ev[1], h->stream);
    int rc = spj_plan_execute(h->plan, col[0], col[1], h->d_out, h->d_n, h->stream);
    if (rc) return rc;
    if (h->events) cudaEventRecord(h->ev[2], h->stream);
    cudaError_t e = cudaMemcpyAsync(h->h_n, h->d_n, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_error(e, "count copy");
    h->started = true;
    return SPJ_OK;
}

int spj_finish(spj_handle_t *h, spj_result_t *out) {
    if (!h || !out) return set_error(SPJ_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    if (!h->started) return set_error(SPJ_E_STATE, "spj_start must precede spj_finish");
    h->started = false;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_error(e, "join execution");
    spj_stats_t st;
    int rc = spj_plan_stats(h->plan, &st);
    if (rc) return rc;
    const int64_t n = *h->h_n;
    if (n < 0 || n > h->h_out_cap) return set_error(SPJ_E_OVERFLOW, "result larger than the host buffer");
    if (n > 0) {
        e = cudaMemcpyAsync(h->h_out, h->d_out, (size_t)n * 8, cudaMemcpyDeviceToHost, h->stream);
        if (e != cudaSuccess) return cuda_error(e, "result copy");
    }
    if (h->events) cudaEventRecord(h->ev[3], h->stream);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_error(e, "result copy");
    h->n_pairs = n;
    // ResultBuffers_t framing (include/type_defs.hpp:82): one contiguous slice per rank
    h->rank_off.assign(h->ranks + 1, 0);
    for (int r = 0; r <= h->ranks; r++) h->rank_off[r] = n * r / h->ranks;
    if (h->events) {
        float a = 0;
        cudaEventElapsedTime(&a, h->ev[0], h->ev[1]);
        h->h2d_ms = a;
        cudaEventElapsedTime(&a, h->ev[2], h->ev[3]);
        h->d2h_ms = a;
    }
    out->pairs = h->h_out;
    out->n_pairs = n;
    out->num_rank = h->ranks;
    out->rank_offsets = h->rank_off.data();
    return SPJ_OK;
}

int spj_record_logs(spj_handle_t *h, spj_stats_t *out, int print) {
    if (!h) return set_error(SPJ_E_ARG, "handle is NULL");
    if (!h->plan) return set_error(SPJ_E_STATE, "no join has run");
    spj_stats_t st;
    int rc = spj_plan_stats(h->plan, &st);
    st.h2d_ms = h->h2d_ms;
    st.d2h_ms = h->d2h_ms;
    if (h->events) {
        float a = 0;
        cudaEventElapsedTime(&a, h->ev[0], h->ev[3]);
        st.total_ms = a;
    }
    if (out) *out = st;
    if (print) {
        // one line per phase, in the spirit of RecordLogs (src/queryHostFunc.cc:183-303)
        printf("phase h2d %.3f ms\nphase partition %.3f ms\nphase join %.3f ms\nphase finish %.3f ms\n"
               "phase d2h %.3f ms\ntotal %.3f ms pairs %lld units %lld radix_bits %d\n",
               st.h2d_ms, st.partition_ms, st.join_ms, st.finish_ms, st.d2h_ms, st.total_ms, (long long)st.n_pairs,
               (long long)st.units, st.radix_bits);
        fflush(stdout);
    }
    return rc;
}

void spj_destroy(spj_handle_t *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_buffers(h);
    cudaFreeHost(h->h_out);
    cudaFreeHost(h->h_n);
    cudaFree(h->d_n);
    if (h->events)
        for (auto &ev : h->ev) cudaEventDestroy(ev);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
