// spj_plan.cu -- host side of libspidjoin: the device-resident plan, the
// JoinInstance-shaped handle of the C ABI, the synthetic-data generator and the
// error reporting. No CPU join path exists: every join runs on the GPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "spj_internal.h"

namespace spj {

cudaError_t launch_pipeline(spj_plan *pl, cudaStream_t st);
cudaError_t configure_kernels(int table_slots, int alg, int *join_blocks_per_sm);
cudaError_t launch_checksum(const spj_kv_pair_t *pairs, const int64_t *n_dev, uint64_t *sum_dev, int sms,
                            cudaStream_t st);
cudaError_t launch_generate(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r,
                            spj_kv_pair_t *s, uint64_t *expect, int sms, cudaStream_t st);
cudaError_t launch_hist_single(const spj_kv_pair_t *t, int64_t n, int bits, uint32_t *hist, int sms,
                               cudaStream_t st);

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    return set_error(e == cudaErrorMemoryAllocation ? SPJ_E_NOMEM : SPJ_E_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

#define SPJ_CUDA(call)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_error(e_, #call); \
    } while (0)

static int ceil_log2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) b++;
    return b;
}

static bool is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

// Checks that a usable sm_100 device is current and returns its SM count.
static int device_sms(int *sms, int *dev_out) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    int dev = 0;
    SPJ_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    SPJ_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return set_error(SPJ_E_NODEVICE, std::string("libspidjoin is built for sm_100a; device is ") + prop.name);
    *sms = prop.multiProcessorCount;
    if (dev_out) *dev_out = dev;
    return SPJ_OK;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace spj

using namespace spj;

extern "C" {

const char *spj_last_error(void) { return g_last_error.c_str(); }

const char *spj_version(void) { return "spidjoin-b200 0.1 (sm_100a)"; }

void spj_design_default(spj_design_t *d) {
    if (!d) return;
    memset(d, 0, sizeof(*d));
    d->input_size = 500000;  // include/idpHandler.hpp:133-138
    d->rank_num = 16;
    d->zipf_factor = 0;
    d->rs_ratio = 8;
    d->rank_set = 1;
    d->bank_set = 1;
    d->tpch_example = 0;
    d->join_alg = SPJ_ALG_PHJ;
    d->radix_bits = 0;
    d->skew_mode = SPJ_SKEW_ADAPTIVE;
    d->unit_tuples = 0;
    d->heavy_sample = 0;
    d->table_slots = 0;
}

static int validate_design(const spj_design_t *d) {
    if (!d) return set_error(SPJ_E_ARG, "design is NULL");
    if (d->rank_num < 1) return set_error(SPJ_E_ARG, "rank_num must be >= 1");
    if (d->rank_set < 1 || d->rank_num % d->rank_set != 0)
        return set_error(SPJ_E_ARG, "rank_set must divide rank_num");
    if (!is_pow2(d->bank_set) || d->bank_set > 64) return set_error(SPJ_E_ARG, "bank_set must be a power of two <= 64");
    if (d->tpch_example) return set_error(SPJ_E_UNSUPPORTED, "tpch_example is not part of the join path");
    if (d->join_alg < SPJ_ALG_PHJ || d->join_alg > SPJ_ALG_NL)
        return set_error(SPJ_E_ARG, "join_alg must be 0 (phj), 1 (nphj), 2 (smj) or 3 (nl)");
    if (d->skew_mode != SPJ_SKEW_ADAPTIVE && d->skew_mode != SPJ_SKEW_FIXED)
        return set_error(SPJ_E_ARG, "skew_mode must be 0 (adaptive) or 1 (fixed)");
    if (d->radix_bits < 0 || d->radix_bits > kMaxRadixBits)
        return set_error(SPJ_E_ARG, "radix_bits must be in [0, 15]");
    if (d->table_slots < 0 || d->unit_tuples < 0) return set_error(SPJ_E_ARG, "negative tuning value");
    return SPJ_OK;
}

int spj_plan_create(int64_t n_r, int64_t n_s, const spj_design_t *design, spj_plan_t **out) {
    if (!out) return set_error(SPJ_E_ARG, "out is NULL");
    *out = nullptr;
    int rc = validate_design(design);
    if (rc) return rc;
    if (n_r < 0 || n_s < 0 || n_r >= 0xFFFFFFFFll || n_s >= 0xFFFFFFFFll)
        return set_error(SPJ_E_ARG, "relation sizes must be in [0, 2^32 - 1)");
    int sms = 0, dev = 0;
    if ((rc = device_sms(&sms, &dev))) return rc;

    spj_plan *pl = new spj_plan();
    pl->n_r = n_r;
    pl->n_s = n_s;
    pl->design = *design;
    pl->device = dev;
    pl->num_sms = sms;
    JoinParams &jp = pl->jp;
    const spj_design_t &d = *design;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int max_slots = (max_smem - 4096) / 8 & ~1;
    int ts = d.table_slots > 0 ? std::min(d.table_slots, max_slots) : kDefaultTableSlots;
    if (d.radix_bits > 0) {
        jp.bits = d.radix_bits;
    } else {
        // Mean R partition at a third of the table (short linear-probe runs), at
        // least 8 partitions per SM for small joins, and at least 64 per rank.
        const uint64_t target = std::max<uint64_t>(1, (uint64_t)ts / 3);
        const int need = ceil_log2((uint64_t)std::max<int64_t>(1, (n_r + target - 1) / target));
        const int par = ceil_log2((uint64_t)8 * sms);
        const int minb = ceil_log2((uint64_t)64 * d.rank_num);
        jp.bits = std::min(std::max(std::max(need, par), minb), kMaxRadixBits);
    }
    if (d.table_slots <= 0) {
        // shrink the table to three times a generous bound on the largest partition
        const double mean = (double)n_r / (double)(1ull << jp.bits);
        const double bound = mean + 6.0 * sqrt(mean) + 32.0;
        const int want = (int)std::min<double>(max_slots, std::max(1024.0, 3.0 * bound));
        ts = std::min(ts, (want + 255) / 256 * 256);
        ts = std::max(ts, 1024);
    }
    jp.table_slots = ts & ~1;  // pairs of slots are probed together
    jp.fine_bits = jp.bits > kMaxPassBits ? jp.bits - (jp.bits + 1) / 2 : 0;
    jp.alg = d.join_alg;
    jp.skew_mode = d.skew_mode;
    jp.group = d.rank_set * d.bank_set;
    jp.unit_tuples = d.unit_tuples > 0 ? (uint32_t)d.unit_tuples : (uint32_t)kDefaultUnitTuples;
    jp.keep_unmatched = (d.join_alg == SPJ_ALG_SMJ || d.join_alg == SPJ_ALG_NL) ? 1 : 0;

    int per_sm = 0;
    cudaError_t ce = configure_kernels(jp.table_slots, jp.alg, &per_sm);
    if (ce != cudaSuccess || per_sm < 1) {
        delete pl;
        return ce != cudaSuccess ? cuda_error(ce, "configure kernels")
                                 : set_error(SPJ_E_ARG, "table_slots too large for one CTA");
    }
    pl->join_blocks = std::min(per_sm * sms, kMaxHoles / (kJoinThreads / 32));

    const uint64_t F = 1ull << jp.bits;
    const int64_t ns[2] = {n_r, n_s};
    // One chunk size for both relations so every pass-1 CTA does the same work;
    // about one wave of 3 CTAs per SM.
    uint32_t nch[2], chunk[2];
    {
        const int64_t total = n_r + n_s;
        int64_t c = std::max<int64_t>(4096, (total + 2 * sms - 3) / (2 * sms - 2));
        c = (c + 1) & ~1ll;
        for (int r = 0; r < 2; r++) {
            nch[r] = (uint32_t)std::max<int64_t>(1, (ns[r] + c - 1) / c);
            chunk[r] = (uint32_t)c;
        }
    }
    // pass-2 work items of ~1/32 of a CTA's share of the tuples
    const uint64_t f1 = 1ull << (jp.bits - jp.fine_bits);
    pl->item_target = (uint32_t)std::max<int64_t>(16384, (n_r + n_s) / (64 * sms));
    const uint64_t max_items = jp.fine_bits ? (uint64_t)(nch[0] + nch[1]) * f1 + 2 * f1 : 1;
    const uint64_t max_units = F * (uint64_t)std::max(jp.group, 1) + (uint64_t)n_s / jp.unit_tuples + F + 64;
    const uint64_t out_cap = (uint64_t)n_s + (uint64_t)pl->join_blocks * (kJoinThreads / 32) * kOutChunk;

    // one arena for all scratch
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    const size_t o_ctr = take(sizeof(Counters));
    const size_t o_hist0 = take((size_t)nch[0] * F * 4), o_hist1 = take((size_t)nch[1] * F * 4);
    const size_t o_ch0 = take((size_t)nch[0] * f1 * 4), o_ch1 = take((size_t)nch[1] * f1 * 4);
    const size_t o_items = take(max_items * 16);
    const size_t o_tot0 = take(F * 4), o_tot1 = take(F * 4), o_base0 = take(F * 4), o_base1 = take(F * 4);
    const bool nphj = jp.alg == SPJ_ALG_NPHJ;
    const size_t o_pr = take(nphj ? 0 : (size_t)n_r * 8 + 16), o_ps = take(nphj ? 0 : (size_t)n_s * 8 + 16);
    if (nphj) {
        uint64_t slots = 1024;
        while (slots < 2 * (uint64_t)n_r) slots <<= 1;
        pl->gtable_slots = slots;
    }
    const size_t o_gt = take(nphj ? pl->gtable_slots * 8 : 0);
    const bool two = !nphj && jp.fine_bits > 0;
    const size_t o_tr = two ? take((size_t)n_r * 8 + 16) : 0, o_ts = two ? take((size_t)n_s * 8 + 16) : 0;
    const size_t o_units = take(max_units * sizeof(Unit));
    const size_t o_holes = take(kMaxHoles * sizeof(Hole));
    const size_t o_gaps = take(kMaxHoles * sizeof(Hole)), o_datas = take(kMaxHoles * sizeof(Hole));
    const size_t o_goff = take(kMaxHoles * 8), o_doff = take(kMaxHoles * 8);
    ce = cudaMalloc(&pl->arena, off);
    if (ce != cudaSuccess) {
        delete pl;
        return cuda_error(ce, "cudaMalloc(plan scratch)");
    }
    pl->arena_bytes = off;
    char *a = (char *)pl->arena;
    PlanDev &P = pl->dev;
    P.ctr = (Counters *)(a + o_ctr);
    for (int r = 0; r < 2; r++) {
        P.rel[r].in = nullptr;
        P.rel[r].n = (uint32_t)ns[r];
        P.rel[r].chunk = chunk[r];
        P.rel[r].nchunks = nch[r];
    }
    P.rel[0].hist = (uint32_t *)(a + o_hist0);
    P.rel[1].hist = (uint32_t *)(a + o_hist1);
    P.rel[0].chist = (uint32_t *)(a + o_ch0);
    P.rel[1].chist = (uint32_t *)(a + o_ch1);
    P.items = (uint4 *)(a + o_items);
    P.max_items = (uint32_t)std::min<uint64_t>(max_items, 0xFFFFFFFFull);
    P.rel[0].total = (uint32_t *)(a + o_tot0);
    P.rel[1].total = (uint32_t *)(a + o_tot1);
    P.rel[0].base = (uint32_t *)(a + o_base0);
    P.rel[1].base = (uint32_t *)(a + o_base1);
    P.rel[0].out = (Tuple *)(a + o_pr);
    P.rel[1].out = (Tuple *)(a + o_ps);
    P.rel[0].tmp = two ? (Tuple *)(a + o_tr) : nullptr;
    P.rel[1].tmp = two ? (Tuple *)(a + o_ts) : nullptr;
    P.units = (Unit *)(a + o_units);
    P.max_units = (uint32_t)std::min<uint64_t>(max_units, 0xFFFFFFFFull);
    P.holes = (Hole *)(a + o_holes);
    P.gaps = (Hole *)(a + o_gaps);
    P.datas = (Hole *)(a + o_datas);
    P.gap_off = (unsigned long long *)(a + o_goff);
    P.data_off = (unsigned long long *)(a + o_doff);
    P.out = nullptr;
    P.out_cap = out_cap;
    P.gtable = nphj ? (unsigned long long *)(a + o_gt) : nullptr;
    P.n_out_user = nullptr;
    pl->have_events = true;
    for (int i = 0; i < spj_plan::kRing && pl->have_events; i++)
        for (int j = 0; j < spj_plan::kMarks; j++)
            if (cudaEventCreate(&pl->ring[i][j]) != cudaSuccess) pl->have_events = false;
    *out = pl;
    return SPJ_OK;
}

int64_t spj_plan_output_capacity(const spj_plan_t *plan) { return plan ? (int64_t)plan->dev.out_cap : 0; }

int spj_plan_execute(spj_plan_t *pl, const spj_kv_pair_t *r, const spj_kv_pair_t *s, spj_kv_pair_t *out,
                     int64_t *n_out, void *stream) {
    if (!pl) return set_error(SPJ_E_ARG, "plan is NULL");
    if ((pl->n_r && !r) || (pl->n_s && !s) || !out) return set_error(SPJ_E_ARG, "NULL column or output");
    if (((uintptr_t)r & 15) || ((uintptr_t)s & 15) || ((uintptr_t)out & 7))
        return set_error(SPJ_E_ARG, "columns must be 16-byte aligned and the output 8-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    PlanDev &P = pl->dev;
    P.rel[0].in = reinterpret_cast<const Tuple *>(r);
    P.rel[1].in = reinterpret_cast<const Tuple *>(s);
    P.out = reinterpret_cast<Tuple *>(out);
    P.n_out_user = reinterpret_cast<unsigned long long *>(n_out);
    SPJ_CUDA(cudaMemsetAsync(P.ctr, 0, sizeof(Counters), st));
    cudaError_t e = launch_pipeline(pl, st);
    if (e != cudaSuccess) return cuda_error(e, "join kernels");
    return SPJ_OK;
}

int spj_plan_stats(spj_plan_t *pl, spj_stats_t *out) {
    if (!pl || !out) return set_error(SPJ_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    Counters c;
    SPJ_CUDA(cudaMemcpy(&c, pl->dev.ctr, sizeof(c), cudaMemcpyDeviceToHost));
    spj_kernel_times_t kt;
    if (pl->have_events && pl->ring_filled > 0 && spj_plan_kernel_times(pl, 0, &kt) == SPJ_OK) {
        out->partition_ms = kt.hist_ms + kt.scan_ms + kt.scatter_ms;
        out->join_ms = kt.units_ms + kt.join_ms;
        out->finish_ms = kt.fixup_ms;
        out->total_ms = kt.total_ms;
    }
    out->n_pairs = (int64_t)c.n_out;
    out->units = c.unit_count;
    out->heavy_keys = c.heavy_keys;
    out->heavy_tuples = (int64_t)c.heavy_tuples;
    out->max_r_partition = c.max_r_part;
    out->max_s_partition = c.max_s_part;
    out->radix_bits = pl->jp.bits;
    out->table_slots = pl->jp.table_slots;
    if (c.error & 32u) return set_error(SPJ_E_TIMEOUT, "a bulk copy did not complete in time");
    if (c.error & 1u)
        return set_error(SPJ_E_OVERFLOW, "an R partition (" + std::to_string(c.max_r_part) +
                                              " tuples) did not fit the shared-memory table of " +
                                              std::to_string(pl->jp.table_slots) + " slots");
    if (c.error)
        return set_error(SPJ_E_OVERFLOW, "internal capacity exceeded (flags " + std::to_string(c.error) + ")");
    return SPJ_OK;
}

int spj_plan_kernel_times(spj_plan_t *pl, int back, spj_kernel_times_t *out) {
    if (!pl || !out) return set_error(SPJ_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    if (!pl->have_events) return set_error(SPJ_E_UNSUPPORTED, "events unavailable");
    if (back < 0 || back >= pl->ring_filled) return set_error(SPJ_E_ARG, "no such execution in the ring");
    const int slot = ((pl->ring_next - 1 - back) % spj_plan::kRing + spj_plan::kRing) % spj_plan::kRing;
    cudaEvent_t *ev = pl->ring[slot];
    SPJ_CUDA(cudaEventSynchronize(ev[spj_plan::kMarks - 1]));
    float t[spj_plan::kMarks - 1];
    for (int i = 0; i + 1 < spj_plan::kMarks; i++) SPJ_CUDA(cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
    out->hist_ms = t[0];
    out->scan_ms = t[1];
    out->scatter_ms = t[2];
    out->units_ms = t[3];
    out->join_ms = t[4];
    out->fixup_ms = t[5];
    float tot = 0;
    SPJ_CUDA(cudaEventElapsedTime(&tot, ev[0], ev[spj_plan::kMarks - 1]));
    out->total_ms = tot;
    return SPJ_OK;
}

void spj_plan_destroy(spj_plan_t *pl) {
    if (!pl) return;
    if (pl->have_events)
        for (auto &row : pl->ring)
            for (auto &e : row)
                if (e) cudaEventDestroy(e);
    cudaFree(pl->arena);
    delete pl;
}

int spj_partition_histogram(const spj_kv_pair_t *tuples, int64_t n, int bits, uint32_t *hist, void *stream) {
    if (bits < 0 || bits > 24 || !hist || (n > 0 && !tuples)) return set_error(SPJ_E_ARG, "bad histogram arguments");
    int sms = 0, rc = device_sms(&sms, nullptr);
    if (rc) return rc;
    cudaError_t e = launch_hist_single(tuples, n, bits, hist, sms, (cudaStream_t)stream);
    return e ? cuda_error(e, "histogram kernel") : SPJ_OK;
}

int spj_checksum_device(const spj_kv_pair_t *pairs, const int64_t *n_dev, uint64_t *sum_dev, void *stream) {
    if (!n_dev || !sum_dev) return set_error(SPJ_E_ARG, "NULL argument");
    int sms = 0, rc = device_sms(&sms, nullptr);
    if (rc) return rc;
    cudaError_t e = launch_checksum(pairs, n_dev, sum_dev, sms, (cudaStream_t)stream);
    return e ? cuda_error(e, "checksum kernel") : SPJ_OK;
}

int spj_generate_device(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r, spj_kv_pair_t *s,
                        uint64_t *expected_checksum_dev, void *stream) {
    if (n_r <= 0 || n_s < 0 || n_r >= 0xFFFFFFFFll || zipf_s < 0) return set_error(SPJ_E_ARG, "bad generator sizes");
    int sms = 0, rc = device_sms(&sms, nullptr);
    if (rc) return rc;
    cudaError_t e = launch_generate(seed, n_r, n_s, zipf_s, r, s, expected_checksum_dev, sms, (cudaStream_t)stream);
    return e ? cuda_error(e, "generator kernels") : SPJ_OK;
}

int spj_generate_host(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r, spj_kv_pair_t *s,
                      uint64_t *expected_checksum, int nthreads) {
    if (n_r <= 0 || n_s < 0 || n_r >= 0xFFFFFFFFll || zipf_s < 0) return set_error(SPJ_E_ARG, "bad generator sizes");
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    const Perm pr = make_perm((uint64_t)n_r, seed_R(seed));
    const Perm prank = make_perm((uint64_t)n_r, seed_rank(seed));
    const GenSpec g{seed, (uint64_t)n_r, (uint64_t)n_s, zipf_s};
    const Zipf z = make_zipf((uint64_t)n_r, zipf_s > 0 ? zipf_s : 1.0);
    std::vector<uint64_t> part(nthreads, 0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) {
        th.emplace_back([&, t]() {
            if (r) {
                int64_t b = n_r * t / nthreads, e = n_r * (t + 1) / nthreads;
                for (int64_t i = b; i < e; i++) {
                    Tuple x = gen_r(pr, (uint64_t)i);
                    r[i].lvalue = x.key;
                    r[i].rvalue = x.pay;
                }
            }
            int64_t b = n_s * t / nthreads, e = n_s * (t + 1) / nthreads;
            uint64_t acc = 0;
            for (int64_t j = b; j < e; j++) {
                uint64_t row = gen_s_row(g, z, prank, (uint64_t)j);
                if (s) {
                    s[j].lvalue = (uint32_t)(1 + perm_apply(pr, row));
                    s[j].rvalue = (uint32_t)j;
                }
                acc += pair_digest((uint32_t)row, (uint32_t)j);
            }
            part[t] = acc;
        });
    }
    for (auto &x : th) x.join();
    if (expected_checksum) {
        uint64_t sum = 0;
        for (uint64_t v : part) sum += v;
        *expected_checksum = sum;
    }
    return SPJ_OK;
}

}  // extern "C"
