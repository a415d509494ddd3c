// spj_plan.cu -- host side of libspidjoin: plans (one join or a batch), their
// device layout, the synthetic-data generator and the error reporting. No CPU
// join path exists: every join runs on the GPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "spj_internal.h"

namespace spj {

cudaError_t launch_checksum(const spj_kv_pair_t *pairs, const int64_t *n_dev, uint64_t *sum_dev, int sms,
                            cudaStream_t st);
cudaError_t launch_generate(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r,
                            spj_kv_pair_t *s, uint64_t *expect, int sms, cudaStream_t st);
cudaError_t launch_hist_single(const spj_kv_pair_t *t, int64_t n, int bits, uint32_t *hist, int sms,
                               cudaStream_t st);
cudaError_t launch_select(const spj_kv_pair_t *in, int64_t n, const spj_predicate_t &p, spj_kv_pair_t *out,
                          int64_t *n_out, int sms, cudaStream_t st);

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    return set_error(e == cudaErrorMemoryAllocation ? SPJ_E_NOMEM : SPJ_E_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

#define SPJ_CUDA(call)                                       \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_error(e_, #call); \
    } while (0)

static int ceil_log2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) b++;
    return b;
}

static bool is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

// Checks that a usable sm_100 device is current and returns its SM count.
// Attribute queries only (cudaGetDeviceProperties costs milliseconds, and this
// runs on every plan creation and every served request).
static int device_sms(int *sms, int *dev_out) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    int dev = 0, major = 0;
    SPJ_CUDA(cudaGetDevice(&dev));
    SPJ_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) {
        cudaDeviceProp prop;
        SPJ_CUDA(cudaGetDeviceProperties(&prop, dev));
        return set_error(SPJ_E_NODEVICE, std::string("libspidjoin is built for sm_100a; device is ") + prop.name);
    }
    SPJ_CUDA(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev));
    if (dev_out) *dev_out = dev;
    return SPJ_OK;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int max_table_slots(int dev) {
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return max_table_slots_for(max_smem);
}

// ------------------------------------------------------------------ tuning --
// The autotuner's per-size-class table (spj_tuning_set): a class is
// (floor(log2 |R|), floor(log2(|S| / |R|)) clamped to [0, 6]).
static std::mutex g_tuning_mu;
static std::vector<spj_tuning_t> g_tuning;

static int log2_floor(uint64_t v) {
    int b = 0;
    while (v > 1) {
        v >>= 1;
        b++;
    }
    return b;
}

const spj_tuning_t *find_tuning(int64_t n_r, int64_t n_s, spj_tuning_t *out) {
    const int lr = log2_floor((uint64_t)std::max<int64_t>(1, n_r));
    const int lt = std::min(6, log2_floor((uint64_t)std::max<int64_t>(1, n_s / std::max<int64_t>(1, n_r))));
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    for (const auto &t : g_tuning)
        if (t.log2_r == lr && t.log2_ratio == lt) {
            *out = t;
            return out;
        }
    return nullptr;
}

// Per-join tuning: the planner's choice for these sizes (size classes follow
// from the formulas: fan-out from |R|, chunking from |R|+|S|).
JoinShape plan_shape(int64_t n_r, int64_t n_s, const spj_design_t &d, int sms, int max_slots, bool alone,
                     int64_t batch_tuples, const spj_tuning_t *tune) {
    JoinShape sh;
    // the local-join algorithm: the design's, or the autotuner's choice for the
    // size class among the algorithms with the same output (the hash joins drop
    // unmatched S tuples, sort-merge and nested loop keep them)
    int alg = d.join_alg;
    // A hash join planned alone whose R's global table (2 to 4 slots of 8 bytes
    // per R tuple, a power of two: at most 64 MiB) fits in half of the 126 MB L2
    // runs as the non-partitioned hash join: same output, no partitioning passes,
    // and its probes hit L2 (|R| <= 2^22 here; measured on B200 it beats the partitioned
    // join there by 1.2-1.6x, and loses from 2^23 on). Adaptive skew mode only:
    // the rank-set and bank-set replication knobs of the fixed mode shape
    // partitions.
    if (alone && alg == SPJ_ALG_PHJ && d.skew_mode == SPJ_SKEW_ADAPTIVE && d.radix_bits <= 0 && n_r > 0 &&
        n_r <= (1 << 22))
        alg = SPJ_ALG_NPHJ;
    if (tune && tune->join_alg > 0) {
        const int ta = tune->join_alg - 1;
        const bool drops = alg == SPJ_ALG_PHJ || alg == SPJ_ALG_NPHJ;
        if (drops == (ta == SPJ_ALG_PHJ || ta == SPJ_ALG_NPHJ)) alg = ta;
    }
    sh.alg = alg;
    const bool tuned_ts = d.table_slots <= 0 && tune && tune->table_slots > 0;
    // a tuned table stays within the default size: in a batch the largest table
    // sets the shared memory, and so the CTAs per SM, of every join kernel
    int ts = d.table_slots > 0 ? std::min(d.table_slots, max_slots)
             : tuned_ts        ? std::min(std::min(tune->table_slots, kDefaultTableSlots), max_slots)
                               : kDefaultTableSlots;
    if (alg == SPJ_ALG_NPHJ) {
        sh.bits = 0;
        sh.fine_bits = 0;
        sh.table_slots = 2;
        // the global table at a load of at most 1/2, or 1/4 while that still keeps
        // it within 32 MiB (|R| <= 2^20): fewer collisions make both the
        // compare-and-swap build and the probe shorter (C1: 0.106 -> 0.081 ms)
        unsigned long long slots = 1024;
        while (slots < (n_r <= (1 << 20) ? 4ull : 2ull) * (unsigned long long)n_r) slots <<= 1;
        sh.gtable_slots = slots;
    } else {
        if (d.radix_bits > 0) {
            sh.bits = d.radix_bits;
        } else {
            // Mean R partition at a third of the table (short linear-probe runs), at
            // least 64 partitions per rank, and -- for a join that runs alone --
            // at least 8 partitions per SM so that a small join still fills the GPU
            // (in a batch the other joins do).
            // (the sort-merge join sorts each R partition in shared memory: half
            // as large partitions keep its sort in a power of two below the table)
            const uint64_t target = std::max<uint64_t>(1, (uint64_t)ts / (alg == SPJ_ALG_SMJ ? 6 : 3));
            const int need = ceil_log2((uint64_t)std::max<int64_t>(1, (n_r + target - 1) / target));
            const int par = alone ? ceil_log2((uint64_t)8 * sms) : 0;
            const int minb = ceil_log2((uint64_t)64 * d.rank_num);
            const int delta = tune ? tune->radix_bits_delta : 0;  // the autotuner's offset for this size class
            sh.bits = std::min(std::max(std::max(std::max(need, par), minb) + delta, 1), kMaxRadixBits);
        }
        if (d.table_slots <= 0 && !tuned_ts) {
            // shrink the table to three times a generous bound on the largest
            // partition (the hash table at a load of 1/3); the sort-merge join
            // wants twice the bound's power of two (its merge sort's two buffers)
            const double mean = (double)n_r / (double)(1ull << sh.bits);
            const double bound = mean + 6.0 * sqrt(mean) + 32.0;
            double pow2 = 1.0;
            while (pow2 < bound) pow2 *= 2.0;
            const double sized = alg == SPJ_ALG_SMJ ? 2.0 * pow2 : 3.0 * bound;
            const int want = (int)std::min<double>(max_slots, std::max(1024.0, sized));
            ts = std::min(ts, (want + 255) / 256 * 256);
            ts = std::max(ts, 1024);
        }
        sh.table_slots = ts & ~1;  // pairs of slots are probed together
        sh.fine_bits = sh.bits > kMaxPassBits ? sh.bits - (sh.bits + 1) / 2 : 0;
    }
    // One chunk size for both relations so every pass-1 CTA does the same work:
    // about one wave of resident scatter CTAs over this join; when the join is
    // one of many, chunks are at least 1/8 wave of the whole batch, so a batch
    // has about eight waves of chunks in all (fine enough to balance the
    // pass-1 CTAs, coarse enough to keep the per-chunk histograms small).
    const int64_t wave = (int64_t)kScatterBlocksPerSM * sms - 2;
    const int64_t spread = std::max<int64_t>(n_r + n_s, batch_tuples / 8);
    int64_t c = std::max<int64_t>(4096, (spread + wave - 1) / wave);
    c = (c + 1) & ~1ll;
    const int64_t ns[2] = {n_r, n_s};
    for (int r = 0; r < 2; r++) {
        sh.nchunks[r] = (uint32_t)std::max<int64_t>(1, (ns[r] + c - 1) / c);
        sh.chunk[r] = (uint32_t)c;
    }
    sh.item_target = (uint32_t)std::max<int64_t>(16384, (n_r + n_s) / (64 * sms));
    // small joins reserve small output chunks, so a batch's output slack stays
    // small; in a batch every warp leaves a hole in each join it touched, so
    // chunks stop at 256 pairs there (a quarter of the fix-up's data to move)
    const uint32_t oc_max = batch_tuples > 0 ? 256u : (uint32_t)kOutChunk;
    uint32_t oc = 32;
    while (oc < oc_max && (int64_t)oc * 8192 < n_s) oc <<= 1;
    sh.out_chunk = oc;
    // Heavy keys joined on the fly: S keys frequent in a sample of S are joined
    // during the first scatter pass (their R payloads found by the count pass
    // over R) and never partitioned. Automatic for the adaptive skew mode when S
    // has at least 2^24 tuples (2^20 in a batch, whose joins are sampled by one
    // launch; a join's own sampling launch costs about as much as the path saves
    // below that): kept only when the heavy keys hold most of the sample;
    // heavy_sample > 0 sets the sample size and keeps whatever heavy keys it
    // finds (in either skew mode); -1 turns the path off.
    if (alg != SPJ_ALG_NPHJ && d.heavy_sample >= 0 && n_s > 0) {
        int64_t hs = 0;
        if (d.heavy_sample > 0) {
            hs = d.heavy_sample;
        } else if (d.skew_mode == SPJ_SKEW_ADAPTIVE && n_s >= (alone ? (1 << 24) : (1 << 20))) {
            hs = kHeavySampleDefault;
            sh.heavy_auto = 1;
        }
        sh.heavy_sample = (uint32_t)std::min<int64_t>(std::min<int64_t>(hs, kHeavySampleMax), n_s);
    }
    sh.unit_tuples = d.unit_tuples > 0                ? (uint32_t)d.unit_tuples
                     : (tune && tune->unit_tuples > 0) ? (uint32_t)tune->unit_tuples
                                                       : (uint32_t)kDefaultUnitTuples;
    if (alg == SPJ_ALG_NPHJ && alone && d.unit_tuples <= 0) {
        // the non-partitioned join's units are plain ranges of S: a join alone
        // cuts S into about eight units per SM so that every SM probes
        const int64_t u = (n_s + 8ll * sms - 1) / (8ll * sms);
        sh.unit_tuples = (uint32_t)std::min<int64_t>(kDefaultUnitTuples, std::max<int64_t>(2048, u));
    }
    return sh;
}

// Arena layout of a plan; with arena == nullptr only the size is computed.
size_t layout_plan(spj_plan *pl, char *a, bool image) {
    const uint32_t J = (uint32_t)pl->joins.size();
    const spj_design_t &d = pl->design;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    const size_t o_ctr = take(sizeof(BatchCtr) + J * sizeof(JoinCtr));
    const size_t o_rel = take(2 * J * sizeof(RelDev)), o_join = take(J * sizeof(JoinDev));
    const size_t o_pref = take((3 * (2 * J + 1) + J + 1) * 4);
    uint64_t max_units = 64, max_items = 1;
    uint32_t tot_chunks = 0, tot_parts = 0, tot_coarse = 0, tot_jparts = 0;
    int max_bits = 0, max_ts = 2, two = 0, any_heavy = 0, alg_mask = 0;
    const uint32_t warps = (uint32_t)pl->join_blocks * (kJoinThreads / 32);
    std::vector<uint32_t> chunk_pref(2 * J + 1), part_pref(2 * J + 1), coarse_pref(2 * J + 1), jpart_pref(J + 1);
    for (uint32_t j = 0; j < J; j++) {
        JoinHost &h = pl->joins[j];
        const JoinShape &sh = pl->shapes[j];
        const bool nphj = sh.alg == SPJ_ALG_NPHJ;
        const uint64_t F = nphj ? 1 : 1ull << sh.bits;
        const uint64_t f1 = (!nphj && sh.fine_bits) ? 1ull << (sh.bits - sh.fine_bits) : 0;
        JoinDev &jd = h.dev;
        Tuple *const bound_out = jd.out;  // pointers bound by the caller survive a re-layout
        unsigned long long *const bound_n = jd.n_out_user;
        jd = JoinDev{};
        jd.out = bound_out;
        jd.n_out_user = bound_n;
        jd.bits = sh.bits;
        jd.fine_bits = nphj ? 0 : sh.fine_bits;
        jd.table_slots = sh.table_slots;
        jd.alg = sh.alg;
        jd.skew_mode = d.skew_mode;
        jd.group = d.rank_set * d.bank_set;
        jd.keep_unmatched = (sh.alg == SPJ_ALG_SMJ || sh.alg == SPJ_ALG_NL) ? 1 : 0;
        jd.unit_tuples = sh.unit_tuples;
        jd.item_target = sh.item_target;
        jd.out_chunk = sh.out_chunk;
        // one output chunk per join warp, plus one for the pairs of heavy keys
        // (their region is rounded up to whole chunks before the join)
        jd.out_cap = (unsigned long long)h.n_s + (unsigned long long)(warps + 1) * sh.out_chunk;
        jd.gtable_slots = nphj ? sh.gtable_slots : 0;
        const int64_t n[2] = {h.n_r, h.n_s};
        for (int r = 0; r < 2; r++) {
            RelDev &rd = h.rel[r];
            const Tuple *const bound_in = rd.in;
            rd = RelDev{};
            rd.in = bound_in;
            rd.n = (uint32_t)n[r];
            const spj_predicate_t &sel = r == 0 ? d.select_r : d.select_s;
            rd.pred = Pred{(uint32_t)sel.field, (uint32_t)sel.op, sel.lo, sel.hi};
            rd.chunk = sh.chunk[r];
            rd.nchunks = nphj ? 0 : sh.nchunks[r];
            rd.join = j;
            const size_t o_hist = take((size_t)rd.nchunks * F * 4);
            const size_t o_chist = take((size_t)rd.nchunks * f1 * 4);
            const size_t o_tot = take(F * 4), o_base = take(F * 4);
            const size_t o_out = take(nphj ? 0 : (size_t)n[r] * 8 + 16);
            const size_t o_tmp = take(f1 ? (size_t)n[r] * 8 + 16 : 0);
            if (a) {
                rd.hist = (uint32_t *)(a + o_hist);
                rd.chist = f1 ? (uint32_t *)(a + o_chist) : nullptr;
                rd.total = (uint32_t *)(a + o_tot);
                rd.base = (uint32_t *)(a + o_base);
                rd.out = nphj ? nullptr : (Tuple *)(a + o_out);
                rd.tmp = f1 ? (Tuple *)(a + o_tmp) : nullptr;
            }
            chunk_pref[2 * j + r] = tot_chunks;
            part_pref[2 * j + r] = tot_parts;
            coarse_pref[2 * j + r] = tot_coarse;
            tot_chunks += rd.nchunks;
            tot_parts += nphj ? 0 : (uint32_t)F;
            tot_coarse += (uint32_t)f1;
        }
        jpart_pref[j] = tot_jparts;
        tot_jparts += nphj ? 1 : (uint32_t)F;
        const size_t o_holes = take(kMaxHoles * sizeof(Hole)), o_gaps = take(kMaxHoles * sizeof(Hole));
        const size_t o_datas = take(kMaxHoles * sizeof(Hole));
        const size_t o_goff = take(kMaxHoles * 8), o_doff = take(kMaxHoles * 8);
        const size_t o_gt = take(nphj ? jd.gtable_slots * 8 : 0);
        const size_t o_hv = take(sh.heavy_sample ? sizeof(HeavyTab) : 0);
        jd.heavy_sample = sh.heavy_sample;
        jd.heavy_auto = sh.heavy_auto;
        if (a) {
            jd.ctr = (JoinCtr *)(a + o_ctr + sizeof(BatchCtr)) + j;
            jd.holes = (Hole *)(a + o_holes);
            jd.gaps = (Hole *)(a + o_gaps);
            jd.datas = (Hole *)(a + o_datas);
            jd.gap_off = (unsigned long long *)(a + o_goff);
            jd.data_off = (unsigned long long *)(a + o_doff);
            jd.gtable = nphj ? (unsigned long long *)(a + o_gt) : nullptr;
            jd.heavy = sh.heavy_sample ? (HeavyTab *)(a + o_hv) : nullptr;
        }
        any_heavy |= sh.heavy_sample ? 1 : 0;
        alg_mask |= 1 << sh.alg;
        max_units += nphj ? (uint64_t)h.n_s / jd.unit_tuples + 64
                          : F * (uint64_t)std::max(jd.group, 1) + (uint64_t)h.n_s / jd.unit_tuples + F + 64;
        if (f1) max_items += (uint64_t)(sh.nchunks[0] + sh.nchunks[1]) * f1 + 2 * f1;
        max_bits = std::max(max_bits, nphj ? 0 : sh.bits);
        max_ts = std::max(max_ts, sh.table_slots);
        two |= f1 ? 1 : 0;
    }
    chunk_pref[2 * J] = tot_chunks;
    part_pref[2 * J] = tot_parts;
    coarse_pref[2 * J] = tot_coarse;
    jpart_pref[J] = tot_jparts;
    const size_t o_units = take(max_units * sizeof(Unit)), o_items = take(max_items * 16);
    if (a) {
        PlanDev &P = pl->dev;
        P.rel = (RelDev *)(a + o_rel);
        P.join = (JoinDev *)(a + o_join);
        uint32_t *pref = (uint32_t *)(a + o_pref);
        P.chunk_prefix = pref;
        P.part_prefix = pref + (2 * J + 1);
        P.coarse_prefix = pref + 2 * (2 * J + 1);
        P.jpart_prefix = pref + 3 * (2 * J + 1);
        P.nrel = 2 * J;
        P.njoin = J;
        P.total_chunks = tot_chunks;
        P.total_parts = tot_parts;
        P.total_coarse = tot_coarse;
        P.total_jparts = tot_jparts;
        P.max_bits = max_bits;
        P.max_table_slots = max_ts;
        P.alg_mask = alg_mask;
        P.any_two_pass = two;
        P.any_heavy = any_heavy;
        P.units = (Unit *)(a + o_units);
        P.max_units = (uint32_t)std::min<uint64_t>(max_units, 0xFFFFFFFFull);
        P.items = (uint4 *)(a + o_items);
        P.max_items = (uint32_t)std::min<uint64_t>(max_items, 0xFFFFFFFFull);
        P.bctr = (BatchCtr *)(a + o_ctr);
        P.jctr = (JoinCtr *)(a + o_ctr + sizeof(BatchCtr));
        pl->desc_offset = o_rel;
    }
    if (a && image) {  // host image of the descriptor region [o_rel, o_pref + prefixes)
        const size_t dend = o_pref + (3 * (2 * J + 1) + J + 1) * 4;
        pl->desc_host.assign(dend - o_rel, 0);
        unsigned char *img = pl->desc_host.data();
        for (uint32_t j = 0; j < J; j++) {
            memcpy(img + (o_rel - o_rel) + (2 * j) * sizeof(RelDev), &pl->joins[j].rel[0], sizeof(RelDev));
            memcpy(img + (2 * j + 1) * sizeof(RelDev), &pl->joins[j].rel[1], sizeof(RelDev));
            memcpy(img + (o_join - o_rel) + j * sizeof(JoinDev), &pl->joins[j].dev, sizeof(JoinDev));
        }
        uint32_t *ip = (uint32_t *)(img + (o_pref - o_rel));
        memcpy(ip, chunk_pref.data(), (2 * J + 1) * 4);
        memcpy(ip + (2 * J + 1), part_pref.data(), (2 * J + 1) * 4);
        memcpy(ip + 2 * (2 * J + 1), coarse_pref.data(), (2 * J + 1) * 4);
        memcpy(ip + 3 * (2 * J + 1), jpart_pref.data(), (J + 1) * 4);
    }
    return off;
}

}  // namespace spj

using namespace spj;

extern "C" {

const char *spj_last_error(void) { return g_last_error.c_str(); }

const char *spj_version(void) { return "spidjoin-b200 0.2 (sm_100a)"; }

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
    for (const spj_predicate_t *p : {&d->select_r, &d->select_s})
        if (p->field < SPJ_PRED_NONE || p->field > SPJ_PRED_PAYLOAD || p->op < SPJ_PRED_EQ || p->op > SPJ_PRED_BETWEEN)
            return set_error(SPJ_E_ARG, "a selection needs field 0..2 (none, key, payload) and op 0..5");
    return SPJ_OK;
}

// Creates a plan of J joins (shared by the plain and the batch entry points).
static int create_plan(int J, const int64_t *n_r, const int64_t *n_s, const spj_design_t *design, spj_plan_t **out) {
    if (!out) return set_error(SPJ_E_ARG, "out is NULL");
    *out = nullptr;
    int rc = validate_design(design);
    if (rc) return rc;
    if (J < 1 || J > 65535) return set_error(SPJ_E_ARG, "a batch holds 1 to 65535 joins");
    for (int j = 0; j < J; j++)
        if (n_r[j] < 0 || n_s[j] < 0 || n_r[j] >= kMaxTuples || n_s[j] >= kMaxTuples)
            return set_error(SPJ_E_ARG, "relation sizes must be in [0, 2^32 - 2^24 - 1)");
    int sms = 0, dev = 0;
    if ((rc = device_sms(&sms, &dev))) return rc;
    spj_plan *pl = new spj_plan();
    pl->n_r = n_r[0];
    pl->n_s = n_s[0];
    pl->design = *design;
    pl->device = dev;
    pl->num_sms = sms;
    const int maxts = max_table_slots(dev);
    pl->joins.resize(J);
    pl->shapes.resize(J);
    int ts_max = 2;
    int64_t batch_tuples = 0;
    if (J > 1)
        for (int j = 0; j < J; j++) batch_tuples += n_r[j] + n_s[j];
    for (int j = 0; j < J; j++) {
        pl->joins[j].n_r = n_r[j];
        pl->joins[j].n_s = n_s[j];
        spj_tuning_t tn;
        pl->shapes[j] = plan_shape(n_r[j], n_s[j], *design, sms, maxts, J == 1, batch_tuples,
                                   J > 1 ? find_tuning(n_r[j], n_s[j], &tn) : nullptr);
        ts_max = std::max(ts_max, pl->shapes[j].table_slots);
    }
    int per_sm = 0, alg_mask = 0;
    for (const JoinShape &sh : pl->shapes) alg_mask |= 1 << sh.alg;
    cudaError_t ce = configure_kernels(ts_max, alg_mask, &per_sm);
    if (ce != cudaSuccess || per_sm < 1) {
        delete pl;
        return ce != cudaSuccess ? cuda_error(ce, "configure kernels")
                                 : set_error(SPJ_E_ARG, "table_slots too large for one CTA");
    }
    pl->join_blocks = std::min(per_sm * sms, kMaxHoles / (kJoinThreads / 32));
    const size_t bytes = layout_plan(pl, nullptr, false);
    ce = cudaMalloc(&pl->arena, bytes);
    if (ce != cudaSuccess) {
        delete pl;
        return cuda_error(ce, "cudaMalloc(plan scratch)");
    }
    pl->arena_bytes = bytes;
    layout_plan(pl, (char *)pl->arena, true);
    // descriptor arrays: uploaded once (a batch's pointers are bound later)
    ce = cudaMemcpy((char *)pl->arena + pl->desc_offset, pl->desc_host.data(), pl->desc_host.size(),
                    cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) {
        cudaFree(pl->arena);
        delete pl;
        return cuda_error(ce, "descriptor upload");
    }
    pl->have_events = true;
    for (int i = 0; i < spj_plan::kRing && pl->have_events; i++)
        for (int k = 0; k < spj_plan::kMarks; k++)
            if (cudaEventCreate(&pl->ring[i][k]) != cudaSuccess) pl->have_events = false;
    *out = pl;
    return SPJ_OK;
}

}  // extern "C"

namespace spj {

// Builds a batch plan whose scratch is allocated stream-ordered on `st` (from
// `pool`, or the device's default pool when it is null), with its column,
// output and per-join count pointers bound and its descriptors uploaded
// asynchronously; no timing events. Used by the join server, whose batches must
// not synchronise the device. *bytes receives the scratch size. Release with
// destroy_plan_stream on the same stream.
int create_plan_stream(int J, const int64_t *n_r, const int64_t *n_s, const spj_design_t *design,
                       const spj_kv_pair_t *const *r, const spj_kv_pair_t *const *s, spj_kv_pair_t *const *out,
                       int64_t *const *n_out, cudaMemPool_t pool, cudaStream_t st, spj_plan_t **pout,
                       size_t *bytes) {
    *pout = nullptr;
    int rc = validate_design(design);
    if (rc) return rc;
    if (J < 1 || J > 65535) return set_error(SPJ_E_ARG, "a batch holds 1 to 65535 joins");
    for (int j = 0; j < J; j++)
        if (n_r[j] < 0 || n_s[j] < 0 || n_r[j] >= kMaxTuples || n_s[j] >= kMaxTuples)
            return set_error(SPJ_E_ARG, "relation sizes must be in [0, 2^32 - 2^24 - 1)");
    int sms = 0, dev = 0;
    if ((rc = device_sms(&sms, &dev))) return rc;
    spj_plan *pl = new spj_plan();
    pl->n_r = n_r[0];
    pl->n_s = n_s[0];
    pl->design = *design;
    pl->device = dev;
    pl->num_sms = sms;
    pl->have_events = false;
    const int maxts = max_table_slots(dev);
    pl->joins.resize(J);
    pl->shapes.resize(J);
    int ts_max = 2;
    int64_t batch_tuples = 0;
    if (J > 1)
        for (int j = 0; j < J; j++) batch_tuples += n_r[j] + n_s[j];
    for (int j = 0; j < J; j++) {
        JoinHost &h = pl->joins[j];
        h.n_r = n_r[j];
        h.n_s = n_s[j];
        spj_tuning_t tn;
        pl->shapes[j] = plan_shape(n_r[j], n_s[j], *design, sms, maxts, J == 1, batch_tuples,
                                   J > 1 ? find_tuning(n_r[j], n_s[j], &tn) : nullptr);
        ts_max = std::max(ts_max, pl->shapes[j].table_slots);
        h.rel[0].in = reinterpret_cast<const Tuple *>(r[j] ? r[j] : out[j]);
        h.rel[1].in = reinterpret_cast<const Tuple *>(s[j] ? s[j] : out[j]);
        h.dev.out = reinterpret_cast<Tuple *>(out[j]);
        h.dev.n_out_user = reinterpret_cast<unsigned long long *>(n_out[j]);
    }
    int per_sm = 0, alg_mask = 0;
    for (const JoinShape &sh : pl->shapes) alg_mask |= 1 << sh.alg;
    cudaError_t ce = configure_kernels(ts_max, alg_mask, &per_sm);
    if (ce != cudaSuccess || per_sm < 1) {
        delete pl;
        return ce != cudaSuccess ? cuda_error(ce, "configure kernels") : set_error(SPJ_E_ARG, "table too large");
    }
    pl->join_blocks = std::min(per_sm * sms, kMaxHoles / (kJoinThreads / 32));
    const size_t b = layout_plan(pl, nullptr, false);
    ce = pool ? cudaMallocFromPoolAsync(&pl->arena, b, pool, st) : cudaMallocAsync(&pl->arena, b, st);
    if (ce != cudaSuccess) {
        delete pl;
        return cuda_error(ce, "stream-ordered allocation of batch scratch");
    }
    pl->arena_bytes = b;
    layout_plan(pl, (char *)pl->arena, true);
    ce = cudaMemcpyAsync((char *)pl->arena + pl->desc_offset, pl->desc_host.data(), pl->desc_host.size(),
                         cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) {
        cudaFreeAsync(pl->arena, st);
        delete pl;
        return cuda_error(ce, "descriptor upload");
    }
    *pout = pl;
    *bytes = b;
    return SPJ_OK;
}

void destroy_plan_stream(spj_plan_t *pl, cudaStream_t st) {
    if (!pl) return;
    cudaFreeAsync(pl->arena, st);
    delete pl;
}

// Output capacity (pairs) a join of these sizes needs inside any plan: |S| plus
// one output chunk per join warp, counting the most join CTAs an SM can hold
// (2048 threads), so no kernel attribute query is needed.
int64_t join_output_capacity(int64_t n_r, int64_t n_s, const spj_design_t &d, bool alone) {
    int sms = 0, dev = 0;
    if (device_sms(&sms, &dev)) return -1;
    spj_tuning_t tn;
    const JoinShape sh = plan_shape(n_r, n_s, d, sms, max_table_slots(dev), alone, 0,
                                    alone ? nullptr : find_tuning(n_r, n_s, &tn));
    const int per_sm = 2048 / kJoinThreads;
    const int blocks = std::min(per_sm * sms, kMaxHoles / (kJoinThreads / 32));
    return n_s + ((int64_t)blocks * (kJoinThreads / 32) + 1) * sh.out_chunk;
}

// Executes a one-join plan; with keep_r, R's partitions from the plan's previous
// execution on the same stream are reused (only S is counted and scattered).
int plan_execute(spj_plan *pl, const spj_kv_pair_t *r, const spj_kv_pair_t *s, spj_kv_pair_t *out, int64_t *n_out,
                 cudaStream_t st, bool keep_r) {
    if (!pl) return set_error(SPJ_E_ARG, "plan is NULL");
    if (pl->joins.size() != 1) return set_error(SPJ_E_ARG, "a batch plan runs with spj_batch_execute");
    if ((pl->n_r && !r) || (pl->n_s && !s) || !out) return set_error(SPJ_E_ARG, "NULL column or output");
    if (((uintptr_t)r & 15) || ((uintptr_t)s & 15) || ((uintptr_t)out & 7))
        return set_error(SPJ_E_ARG, "columns must be 16-byte aligned and the output 8-byte aligned");
    JoinHost &h = pl->joins[0];
    // an empty relation still needs a readable, aligned column pointer
    h.rel[0].in = r ? reinterpret_cast<const Tuple *>(r) : reinterpret_cast<const Tuple *>(out);
    h.rel[1].in = s ? reinterpret_cast<const Tuple *>(s) : reinterpret_cast<const Tuple *>(out);
    h.dev.out = reinterpret_cast<Tuple *>(out);
    h.dev.n_out_user = reinterpret_cast<unsigned long long *>(n_out);
    cudaError_t e = init_single(pl, st, keep_r);  // also zeroes the counters
    if (e != cudaSuccess) return cuda_error(e, "descriptor kernel");
    e = launch_pipeline(pl, st, keep_r);
    if (e != cudaSuccess) return cuda_error(e, "join kernels");
    return SPJ_OK;
}

}  // namespace spj

extern "C" {

int spj_plan_create(int64_t n_r, int64_t n_s, const spj_design_t *design, spj_plan_t **out) {
    return create_plan(1, &n_r, &n_s, design, out);
}

// The same plan_shape call as create_plan, with the device limits as arguments.
int spj_plan_describe(int64_t n_r, int64_t n_s, const spj_design_t *design, int num_sms, int max_smem_per_block,
                      int64_t batch_tuples, spj_plan_shape_t *out) {
    if (!out) return set_error(SPJ_E_ARG, "out is NULL");
    int rc = validate_design(design);
    if (rc) return rc;
    if (n_r < 0 || n_s < 0 || n_r >= kMaxTuples || n_s >= kMaxTuples)
        return set_error(SPJ_E_ARG, "relation sizes must be in [0, 2^32 - 2^24 - 1)");
    if (num_sms < 1 || max_smem_per_block < 48 * 1024 || batch_tuples < 0)
        return set_error(SPJ_E_ARG, "num_sms >= 1, max_smem_per_block >= 48 KiB, batch_tuples >= 0");
    const bool alone = batch_tuples == 0;
    spj_tuning_t tn;
    const JoinShape sh = plan_shape(n_r, n_s, *design, num_sms, max_table_slots_for(max_smem_per_block), alone,
                                    batch_tuples, alone ? nullptr : find_tuning(n_r, n_s, &tn));
    const bool nphj = sh.alg == SPJ_ALG_NPHJ;
    out->join_alg = sh.alg;
    out->radix_bits = nphj ? 0 : sh.bits;
    out->scatter_passes = nphj ? 0 : (sh.fine_bits ? 2 : 1);
    out->table_slots = nphj ? 0 : sh.table_slots;
    out->global_table_slots = nphj ? (int64_t)sh.gtable_slots : 0;
    out->heavy_sample = (int32_t)sh.heavy_sample;
    out->unit_tuples = (int32_t)sh.unit_tuples;
    out->out_chunk = (int32_t)sh.out_chunk;
    out->chunk_tuples = (int32_t)sh.chunk[0];
    return SPJ_OK;
}

int64_t spj_plan_output_capacity(const spj_plan_t *plan) {
    return plan ? (int64_t)plan->joins[0].dev.out_cap : 0;
}

int spj_plan_execute(spj_plan_t *pl, const spj_kv_pair_t *r, const spj_kv_pair_t *s, spj_kv_pair_t *out,
                     int64_t *n_out, void *stream) {
    return plan_execute(pl, r, s, out, n_out, (cudaStream_t)stream, false);
}


static void fill_stats(const spj_plan *pl, const JoinCtr &c, spj_stats_t *out) {
    out->n_pairs = (int64_t)c.n_out;
    out->units = c.units;
    out->max_r_partition = c.max_r_part;
    out->max_s_partition = c.max_s_part;
    out->radix_bits = pl->shapes[0].bits;
    out->table_slots = pl->shapes[0].table_slots;
    out->heavy_keys = c.heavy_keys;
    out->heavy_tuples = (int64_t)c.heavy_tuples;
    out->join_alg = pl->shapes[0].alg;
}

static int ctr_error(const spj_plan *pl, unsigned err, unsigned max_r) {
    if (err & 32u) return set_error(SPJ_E_TIMEOUT, "a bulk copy did not complete in time");
    if (err & 1u)
        return set_error(SPJ_E_OVERFLOW, "an R partition (" + std::to_string(max_r) +
                                              " tuples) did not fit the shared-memory structure of its CTA");
    if (err) return set_error(SPJ_E_OVERFLOW, "internal capacity exceeded (flags " + std::to_string(err) + ")");
    (void)pl;
    return SPJ_OK;
}

int spj_plan_stats(spj_plan_t *pl, spj_stats_t *out) {
    if (!pl || !out) return set_error(SPJ_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    JoinCtr c;
    SPJ_CUDA(cudaMemcpy(&c, pl->dev.jctr, sizeof(c), cudaMemcpyDeviceToHost));
    spj_kernel_times_t kt;
    if (pl->have_events && pl->ring_filled > 0 && spj_plan_kernel_times(pl, 0, &kt) == SPJ_OK) {
        out->partition_ms = kt.hist_ms + kt.scan_ms + kt.scatter_ms;
        out->join_ms = kt.units_ms + kt.join_ms;
        out->finish_ms = kt.fixup_ms;
        out->total_ms = kt.total_ms;
    }
    fill_stats(pl, c, out);
    return ctr_error(pl, c.error, c.max_r_part);
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

// ------------------------------------------------------------------ batches --

int spj_batch_create(int n_joins, const int64_t *n_r, const int64_t *n_s, const spj_design_t *design,
                     spj_plan_t **out) {
    if (!n_r || !n_s) return set_error(SPJ_E_ARG, "NULL size arrays");
    return create_plan(n_joins, n_r, n_s, design, out);
}

int64_t spj_batch_output_capacity(const spj_plan_t *plan, int j) {
    if (!plan || j < 0 || j >= (int)plan->joins.size()) return 0;
    return (int64_t)plan->joins[j].dev.out_cap;
}

int spj_batch_bind(spj_plan_t *pl, const spj_kv_pair_t *const *r, const spj_kv_pair_t *const *s,
                   spj_kv_pair_t *const *out, int64_t *n_out) {
    if (!pl || !r || !s || !out) return set_error(SPJ_E_ARG, "NULL pointer array");
    const size_t J = pl->joins.size();
    for (size_t j = 0; j < J; j++) {
        JoinHost &h = pl->joins[j];
        if ((h.n_r && !r[j]) || (h.n_s && !s[j]) || !out[j]) return set_error(SPJ_E_ARG, "NULL column or output");
        if (((uintptr_t)r[j] & 15) || ((uintptr_t)s[j] & 15) || ((uintptr_t)out[j] & 7))
            return set_error(SPJ_E_ARG, "columns must be 16-byte aligned and outputs 8-byte aligned");
        h.rel[0].in = reinterpret_cast<const Tuple *>(r[j] ? r[j] : out[j]);
        h.rel[1].in = reinterpret_cast<const Tuple *>(s[j] ? s[j] : out[j]);
        h.dev.out = reinterpret_cast<Tuple *>(out[j]);
        h.dev.n_out_user = n_out ? reinterpret_cast<unsigned long long *>(n_out + j) : nullptr;
    }
    layout_plan(pl, (char *)pl->arena, true);  // refreshes the host image with the bound pointers
    SPJ_CUDA(cudaMemcpy((char *)pl->arena + pl->desc_offset, pl->desc_host.data(), pl->desc_host.size(),
                        cudaMemcpyHostToDevice));
    return SPJ_OK;
}

int spj_batch_execute(spj_plan_t *pl, void *stream) {
    if (!pl) return set_error(SPJ_E_ARG, "plan is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    SPJ_CUDA(cudaMemsetAsync(pl->dev.bctr, 0, sizeof(BatchCtr) + pl->joins.size() * sizeof(JoinCtr), st));
    cudaError_t e = launch_pipeline(pl, st);
    if (e != cudaSuccess) return cuda_error(e, "join kernels");
    return SPJ_OK;
}

int spj_batch_stats(spj_plan_t *pl, int j, spj_stats_t *out) {
    if (!pl || !out || j < 0 || j >= (int)pl->joins.size()) return set_error(SPJ_E_ARG, "bad argument");
    memset(out, 0, sizeof(*out));
    JoinCtr c;
    SPJ_CUDA(cudaMemcpy(&c, pl->dev.jctr + j, sizeof(c), cudaMemcpyDeviceToHost));
    fill_stats(pl, c, out);
    out->radix_bits = pl->shapes[j].bits;
    out->table_slots = pl->shapes[j].table_slots;
    out->join_alg = pl->shapes[j].alg;
    return ctr_error(pl, c.error, c.max_r_part);
}

int spj_partition_histogram(const spj_kv_pair_t *tuples, int64_t n, int bits, uint32_t *hist, void *stream) {
    if (bits < 0 || bits > 24 || !hist || (n > 0 && !tuples)) return set_error(SPJ_E_ARG, "bad histogram arguments");
    int sms = 0, rc = device_sms(&sms, nullptr);
    if (rc) return rc;
    cudaError_t e = launch_hist_single(tuples, n, bits, hist, sms, (cudaStream_t)stream);
    return e ? cuda_error(e, "histogram kernel") : SPJ_OK;
}

int spj_select(const spj_kv_pair_t *in, int64_t n, const spj_predicate_t *pred, spj_kv_pair_t *out, int64_t *n_out,
               void *stream) {
    if (!pred || !n_out || n < 0 || (n > 0 && (!in || !out))) return set_error(SPJ_E_ARG, "bad selection arguments");
    if (pred->field < SPJ_PRED_NONE || pred->field > SPJ_PRED_PAYLOAD || pred->op < SPJ_PRED_EQ ||
        pred->op > SPJ_PRED_BETWEEN)
        return set_error(SPJ_E_ARG, "a selection needs field 0..2 (none, key, payload) and op 0..5");
    int sms = 0, rc = device_sms(&sms, nullptr);
    if (rc) return rc;
    cudaError_t e = launch_select(in, n, *pred, out, n_out, sms, (cudaStream_t)stream);
    return e ? cuda_error(e, "selection kernel") : SPJ_OK;
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

namespace spj {
// The status a finished join's counter error bits map to (the message goes to
// the calling thread's last error).
int join_ctr_status(unsigned err, unsigned max_r_part) { return ctr_error(nullptr, err, max_r_part); }
}  // namespace spj

extern "C" {

int spj_tuning_set(const spj_tuning_t *entries, int n) {
    if (n < 0 || (n > 0 && !entries)) return set_error(SPJ_E_ARG, "bad tuning table");
    for (int i = 0; i < n; i++) {
        const spj_tuning_t &t = entries[i];
        if (t.log2_r < 0 || t.log2_r > 32 || t.log2_ratio < 0 || t.log2_ratio > 6 || t.radix_bits_delta < -4 ||
            t.radix_bits_delta > 4 || t.table_slots < 0 || t.unit_tuples < 0 || t.join_alg < 0 || t.join_alg > 4)
            return set_error(SPJ_E_ARG, "tuning entry " + std::to_string(i) + " out of range");
    }
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    g_tuning.assign(entries, entries + n);
    return SPJ_OK;
}

int spj_tuning_get(spj_tuning_t *entries, int capacity) {
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    const int n = (int)g_tuning.size();
    if (entries)
        for (int i = 0; i < n && i < capacity; i++) entries[i] = g_tuning[i];
    return n;
}

}  // extern "C"
