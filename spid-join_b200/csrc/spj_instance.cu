// spj_instance.cu -- the JoinInstance-shaped handle of the C ABI
// (pidjoin::JoinInstance, include/join_internals.hpp:301-323 of yonsei-hpcp/spid-join).
//
// Reference flow: LoadColumn splits and aliases the caller's columns,
// PrepareJoin allocates ranks and spawns one thread per rank, StartJoin signals
// them, FinishJoin joins the threads and returns per-rank result buffers
// (src/query.cc:178-317, 1517-1567); the host moves columns to the DPUs and
// results back (SEND/RECV, src/queryHostFunc.cc:1058-1126, 1421-1498).
//
// Here: load_column borrows the column, prepare builds the device plans and
// buffers, start enqueues the copies and the joins, finish waits and copies
// the pairs back. When S lives in host memory and is large, it is joined in
// slices so that the three streams of an instance overlap: slice i+1 is copied
// to the device while slice i is joined and slice i-1's pairs are copied back
// (the host link carries both directions at once). Every slice joins all of R,
// so the union of the slices' outputs is the join's output. R is partitioned
// once per join: the slices after the first reuse its partitions and count and
// scatter only their own S, so slices can be small and the tail after the last
// input copy (the last slice's join and result copy) short. All slices have
// one length and one plan: the device copy of S is padded to whole slices with
// key-0 tuples, the empty key, which no pass keeps. Instances are independent.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "spj_internal.h"

using namespace spj;

namespace {
constexpr int kMaxSlices = 32;
constexpr int64_t kSliceMin = 1ll << 24;  // host S below this is joined in one piece
// Target S tuples per slice. Every slice's join still builds the tables of all
// of R's partitions (~1.4 ms for 2^27 R tuples), so a slice must carry enough S
// for its upload to cover that: 2^24 tuples (128 MiB, ~2.6 ms of upload).
constexpr int64_t kSliceTuples = 1ll << 24;
}  // namespace

struct spj_handle {
    int ranks = 1, rank_groups = 1, ranks_per_group = 1;
    const void *col[2] = {nullptr, nullptr};
    int64_t n[2] = {0, 0};
    bool col_set[2] = {false, false};
    bool on_device[2] = {false, false};
    spj_design_t design{};
    spj_plan_t *plan = nullptr;  // joins R with one slice
    int nslices = 1;
    int64_t slice = 0;      // S tuples per slice (multiple of 256 when sliced)
    int64_t slice_cap = 0;  // output pairs reserved per slice on the device
    bool started = false;
    bool loaded = false;  // a column was loaded after the last prepare
    cudaStream_t stream = nullptr, s_in = nullptr, s_out = nullptr;  // joins, host->device, device->host
    spj_kv_pair_t *d_col[2] = {nullptr, nullptr};  // device copies of host columns
    spj_kv_pair_t *d_out = nullptr;                // nslices x slice_cap pairs
    int64_t *d_n = nullptr;                        // per-slice pair counts
    int64_t *h_n = nullptr;                        // pinned copies of d_n
    JoinCtr *h_ctr = nullptr;                      // pinned: each slice's counters
    spj_kv_pair_t *h_out = nullptr;                // pinned result
    int64_t h_out_cap = 0;
    int64_t n_pairs = 0;
    std::vector<int64_t> rank_off;
    cudaEvent_t ev[4]{};  // start, all columns on the device, all joins done, all pairs on the host
    cudaEvent_t ev_in[kMaxSlices]{}, ev_done[kMaxSlices]{};
    bool events = false;
    double d2h_ms = 0, h2d_ms = 0;
};

static void free_buffers(spj_handle_t *h) {
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_col[i]);
        h->d_col[i] = nullptr;
    }
    cudaFree(h->d_out);
    h->d_out = nullptr;
    if (h->plan) spj_plan_destroy(h->plan);
    h->plan = nullptr;
    h->nslices = 1;
}

// Host S tuples of slice i (the device copy of a sliced S is padded to whole slices).
static int64_t slice_len(const spj_handle_t *h, int i) {
    return std::max<int64_t>(0, std::min(h->slice, h->n[1] - (int64_t)i * h->slice));
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
    cudaError_t e = cudaSuccess;
    for (cudaStream_t *s : {&h->stream, &h->s_in, &h->s_out})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_n, kMaxSlices * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_ctr, kMaxSlices * sizeof(JoinCtr));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_n, kMaxSlices * sizeof(int64_t));
    for (int i = 0; i < kMaxSlices && e == cudaSuccess; i++) {
        e = cudaEventCreateWithFlags(&h->ev_in[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_done[i], cudaEventDisableTiming);
    }
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
    h->loaded = true;
    return SPJ_OK;
}

int spj_prepare(spj_handle_t *h, const spj_design_t *design) {
    if (!h) return set_error(SPJ_E_ARG, "handle is NULL");
    if (h->started) return set_error(SPJ_E_STATE, "join in flight; call spj_finish first");
    if (!h->col_set[0] || !h->col_set[1]) return set_error(SPJ_E_STATE, "load both columns before prepare");
    h->loaded = false;
    spj_design_t d = design ? *design : h->design;
    // the instance's rank layout is authoritative (JoinInstance(r, R, r/R))
    d.rank_num = h->ranks;
    d.rank_set = h->rank_groups;
    // slicing of a host S (see the file comment)
    int ns = 1;
    if (!h->on_device[1] && h->n[1] >= kSliceMin)
        ns = (int)std::min<int64_t>(kMaxSlices, (h->n[1] + kSliceTuples - 1) / kSliceTuples);
    int64_t slice = h->n[1];
    if (ns > 1) {
        slice = ((h->n[1] + ns - 1) / ns + 255) / 256 * 256;
        ns = (int)((h->n[1] + slice - 1) / slice);
    }
    bool same_copies = true;  // device copies exist exactly for the host columns
    for (int i = 0; i < 2; i++) same_copies &= (h->d_col[i] != nullptr) == (!h->on_device[i] && h->n[i] > 0);
    if (h->plan && same_copies && h->plan->n_r == h->n[0] && h->nslices == ns && h->slice == slice &&
        h->plan->n_s == slice && memcmp(&h->plan->design, &d, sizeof(d)) == 0) {
        h->design = d;
        return SPJ_OK;  // reuse the plans and their buffers
    }
    free_buffers(h);
    h->nslices = ns;
    h->slice = slice;
    int rc = spj_plan_create(h->n[0], slice, &d, &h->plan);
    if (rc) {
        free_buffers(h);
        return rc;
    }
    h->design = d;
    cudaError_t e = cudaSuccess;
    const int64_t s_dev = ns > 1 ? (int64_t)ns * slice : h->n[1];  // device S tuples, padding included
    for (int i = 0; i < 2 && e == cudaSuccess; i++)
        if (!h->on_device[i] && h->n[i] > 0) e = cudaMalloc(&h->d_col[i], (size_t)(i ? s_dev : h->n[0]) * 8);
    h->slice_cap = spj_plan_output_capacity(h->plan);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_out, (size_t)h->slice_cap * ns * 8);
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
    if (h->loaded) {  // columns changed since the last prepare: size the plans for them
        int rc = spj_prepare(h, &h->design);
        if (rc) return rc;
    }
    if (design) {
        spj_design_t d = *design;
        d.rank_num = h->ranks;
        d.rank_set = h->rank_groups;
        if (memcmp(&d, &h->design, sizeof(d)) != 0) {
            int rc = spj_prepare(h, &d);
            if (rc) return rc;
        }
    }
    if (h->events) cudaEventRecord(h->ev[0], h->s_in);
    const spj_kv_pair_t *col[2];
    for (int i = 0; i < 2; i++)
        col[i] = h->n[i] == 0 ? h->d_out  // never read; any aligned device pointer
                              : h->on_device[i] ? (const spj_kv_pair_t *)h->col[i] : h->d_col[i];
    cudaError_t e = cudaSuccess;
    const int64_t s_dev = h->nslices > 1 ? (int64_t)h->nslices * h->slice : h->n[1];
    if (s_dev > h->n[1])  // key-0 padding of the last slice, before its copy on the same stream
        e = cudaMemsetAsync(h->d_col[1] + h->n[1], 0, (size_t)(s_dev - h->n[1]) * 8, h->s_in);
    if (e == cudaSuccess && !h->on_device[0] && h->n[0] > 0)
        e = cudaMemcpyAsync(h->d_col[0], h->col[0], (size_t)h->n[0] * 8, cudaMemcpyHostToDevice, h->s_in);
    for (int i = 0; i < h->nslices && e == cudaSuccess; i++) {
        const int64_t off = (int64_t)i * h->slice, len = slice_len(h, i);
        if (!h->on_device[1] && len > 0)
            e = cudaMemcpyAsync(h->d_col[1] + off, (const spj_kv_pair_t *)h->col[1] + off, (size_t)len * 8,
                                cudaMemcpyHostToDevice, h->s_in);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_in[i], h->s_in);
    }
    if (e == cudaSuccess && h->events) e = cudaEventRecord(h->ev[1], h->s_in);
    if (e != cudaSuccess) return cuda_error(e, "column copy");
    for (int i = 0; i < h->nslices; i++) {
        spj_plan_t *pl = h->plan;
        const int64_t off = (int64_t)i * h->slice;
        e = cudaStreamWaitEvent(h->stream, h->ev_in[i], 0);
        if (e != cudaSuccess) return cuda_error(e, "slice dependency");
        // slice 0 partitions R; the later slices reuse its partitions
        int rc = plan_execute(pl, col[0], h->n[1] ? col[1] + off : col[1], h->d_out + (size_t)i * h->slice_cap,
                              h->d_n + i, h->stream, i > 0);
        if (rc) return rc;
        e = cudaMemcpyAsync(h->h_n + i, h->d_n + i, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h->h_ctr + i, pl->dev.jctr, sizeof(JoinCtr), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_done[i], h->stream);
        if (e != cudaSuccess) return cuda_error(e, "slice completion record");
    }
    if (h->events) cudaEventRecord(h->ev[2], h->stream);
    h->started = true;
    return SPJ_OK;
}

int spj_finish(spj_handle_t *h, spj_result_t *out) {
    if (!h || !out) return set_error(SPJ_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    if (!h->started) return set_error(SPJ_E_STATE, "spj_start must precede spj_finish");
    h->started = false;
    // each slice's pairs go back as soon as that slice's join is done
    int64_t n = 0;
    int rc = SPJ_OK;
    for (int i = 0; i < h->nslices; i++) {
        cudaError_t e = cudaEventSynchronize(h->ev_done[i]);
        if (e != cudaSuccess) return cuda_error(e, "join execution");
        if (rc == SPJ_OK) rc = join_ctr_status(h->h_ctr[i].error, h->h_ctr[i].max_r_part);
        const int64_t ni = h->h_n[i];
        if (rc == SPJ_OK && (ni < 0 || n + ni > h->h_out_cap))
            rc = set_error(SPJ_E_OVERFLOW, "result larger than the host buffer");
        if (rc == SPJ_OK && ni > 0) {
            e = cudaMemcpyAsync(h->h_out + n, h->d_out + (size_t)i * h->slice_cap, (size_t)ni * 8,
                                cudaMemcpyDeviceToHost, h->s_out);
            if (e != cudaSuccess) rc = cuda_error(e, "result copy");
        }
        if (rc == SPJ_OK) n += ni;
    }
    if (h->events) cudaEventRecord(h->ev[3], h->s_out);
    cudaError_t e = cudaStreamSynchronize(h->s_out);
    if (rc) return rc;
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
    int rc = spj_plan_stats(h->plan, &st);  // the last slice's join
    st.n_pairs = h->n_pairs;
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
               "phase d2h %.3f ms\ntotal %.3f ms pairs %lld units %lld radix_bits %d slices %d\n",
               st.h2d_ms, st.partition_ms, st.join_ms, st.finish_ms, st.d2h_ms, st.total_ms, (long long)st.n_pairs,
               (long long)st.units, st.radix_bits, h->nslices);
        fflush(stdout);
    }
    return rc;
}

void spj_destroy(spj_handle_t *h) {
    if (!h) return;
    for (cudaStream_t s : {h->stream, h->s_in, h->s_out})
        if (s) cudaStreamSynchronize(s);
    free_buffers(h);
    cudaFreeHost(h->h_out);
    cudaFreeHost(h->h_n);
    cudaFreeHost(h->h_ctr);
    cudaFree(h->d_n);
    for (int i = 0; i < kMaxSlices; i++) {
        if (h->ev_in[i]) cudaEventDestroy(h->ev_in[i]);
        if (h->ev_done[i]) cudaEventDestroy(h->ev_done[i]);
    }
    if (h->events)
        for (auto &ev : h->ev) cudaEventDestroy(ev);
    for (cudaStream_t s : {h->stream, h->s_in, h->s_out})
        if (s) cudaStreamDestroy(s);
    delete h;
}

}  // extern "C"
