/*
 * spidjoin.h -- C ABI of the B200-native SPID-Join equi-join (libspidjoin.so).
 *
 * The join computes, for relations R (build side) and S (probe side) of 8-byte
 * tuples {u32 key, u32 payload}, the pairs (R.payload, S.payload) of equal keys.
 * Key 0 marks padding and never joins. Every entry point returns SPJ_OK (0) or a
 * negative SPJ_E_* code; spj_last_error() gives the message of the last failure
 * on the calling thread. No entry point exits the process.
 *
 * Each declaration names the interface of the reference (yonsei-hpcp/spid-join,
 * paths relative to that project) that it replaces. The C++ facade in
 * pidjoin.hpp maps the reference's pidjoin::JoinInstance onto these calls.
 */
#ifndef SPIDJOIN_H
#define SPIDJOIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kv_pair_t, include/type_defs.hpp:53-56: lvalue = key, rvalue = payload.
 * Output pairs reuse it as {lvalue = R payload, rvalue = S payload}. */
typedef struct {
    uint32_t lvalue;
    uint32_t rvalue;
} spj_kv_pair_t;

enum spj_status {
    SPJ_OK = 0,
    SPJ_E_ARG = -1,         /* invalid argument or design */
    SPJ_E_NOMEM = -2,       /* host or device allocation failed */
    SPJ_E_CUDA = -3,        /* a CUDA call failed (message has the CUDA error) */
    SPJ_E_STATE = -4,       /* call out of order (e.g. start before prepare) */
    SPJ_E_OVERFLOW = -5,    /* a partition exceeded its shared-memory table */
    SPJ_E_TIMEOUT = -6,     /* a bounded device wait gave up */
    SPJ_E_NODEVICE = -7,    /* no CUDA device, or not an sm_100 device */
    SPJ_E_UNSUPPORTED = -8  /* option this library does not support */
};

/* join_alg values, include/idpHandler.hpp:135-138 */
enum spj_join_alg {
    SPJ_ALG_PHJ = 0,   /* partitioned hash join: at most one match per S tuple,
                          unmatched S tuples dropped (a2a_srj_probe_inner_mt.c:136-148) */
    SPJ_ALG_NPHJ = 1,  /* non-partitioned hash join (global table) */
    SPJ_ALG_SMJ = 2,   /* sort-merge: S rewritten in place, unmatched S kept as is
                          (mpsm_join_sort_probe.c:214-236) */
    SPJ_ALG_NL = 3     /* nested loop over sub-partitions of <= 256 R tuples, S rewritten
                          in place (nested_loop_join.c:184-231) */
};

enum spj_skew_mode {
    SPJ_SKEW_ADAPTIVE = 0, /* heavy partitions split so no work unit exceeds unit_tuples S tuples
                              (at least `group` units each); heavy keys found in a sample of S are
                              joined on the fly (see heavy_sample) */
    SPJ_SKEW_FIXED = 1     /* every heavy partition split into exactly `group` units, the
                              reference's fixed rank-set x bank-set replication */
};

/* A selection applied to a relation before it is joined: the reference's
 * TPC-H-style predicates (src/dpu/include/select.h: the comparison operators of
 * PREDINT64, :30-37, and predi_btw's inclusive range, :44-47) on a tuple's key
 * or payload, as unsigned 32-bit values (the reference compares its dates the
 * same way, predd, :4-11). The join path evaluates them inside its first pass
 * over each relation (count and first scatter, or the non-partitioned join's
 * build and probe), so the filtered tuples are never written; spj_select
 * applies one on its own. */
enum spj_pred_field { SPJ_PRED_NONE = 0, SPJ_PRED_KEY = 1, SPJ_PRED_PAYLOAD = 2 };
enum spj_pred_op {
    SPJ_PRED_EQ = 0,      /* value == lo */
    SPJ_PRED_LE = 1,      /* value <= lo */
    SPJ_PRED_GE = 2,      /* value >= lo */
    SPJ_PRED_LT = 3,      /* value < lo */
    SPJ_PRED_GT = 4,      /* value > lo */
    SPJ_PRED_BETWEEN = 5  /* lo <= value <= hi */
};
typedef struct {
    int field;  /* enum spj_pred_field (SPJ_PRED_NONE: every tuple passes) */
    int op;     /* enum spj_pred_op */
    uint32_t lo, hi;
} spj_predicate_t;

/* join_design_t, include/idpHandler.hpp:131-145, followed by B200 tuning fields
 * (0 = chosen by the planner). rank_num, rank_set and bank_set keep the
 * reference's meaning as replication knobs: 64 * rank_num is the minimum
 * partition fan-out and rank_set * bank_set the replica group of a heavy
 * partition (the CTAs that each build its R table and split its S). */
typedef struct {
    int64_t input_size; /* -s: |R| of the synthetic driver */
    int rank_num;       /* -r */
    int zipf_factor;    /* -z: Zipf exponent x 100 */
    int rs_ratio;       /* -t: |S| / |R| */
    int rank_set;       /* -R */
    int bank_set;       /* -B: any power of two (the reference accepts 1, 8, 16, 32, 64) */
    int tpch_example;   /* unused (must be 0) */
    int join_alg;       /* enum spj_join_alg */
    /* B200 tuning */
    int radix_bits;     /* partition fan-out = 2^radix_bits */
    int skew_mode;      /* enum spj_skew_mode */
    int unit_tuples;    /* max S tuples per work unit in adaptive mode */
    int heavy_sample;   /* S keys sampled to find heavy keys, which the first scatter pass joins
                           on the fly (at most 256 per join; their S tuples skip the
                           partitioning): 0 = 16384 in the adaptive skew mode when |S| >= 2^24
                           (2^20 for a join in a batch),
                           kept only when the heavy keys hold at least 60% of the sample (below
                           that the per-tuple filter lookups cost more than they save), else
                           off; > 0 = that many, kept whatever their share (any skew mode);
                           -1 = off */
    int table_slots;    /* shared-memory hash-table slots per CTA */
    spj_predicate_t select_r, select_s; /* selections on R and S ahead of the join */
    int reserved[4];
} spj_design_t;

/* Fills the reference's defaults (idpHandler.hpp:131-145) and automatic tuning. */
void spj_design_default(spj_design_t *design);

const char *spj_last_error(void);
const char *spj_version(void);

/* ------------------------------------------------------------- instance -- */

typedef struct spj_handle spj_handle_t;

/* JoinInstance(int num_rank_allocated, int num_rankgroup, int num_rank_in_rankgroup),
 * include/join_internals.hpp:306. Binds to the current CUDA device. */
int spj_create(int num_rank_allocated, int num_rankgroup, int num_rank_in_rankgroup, spj_handle_t **out);

/* void LoadColumn(void *data_ptr, int64_t num_tuples, std::string col_name),
 * include/join_internals.hpp:316; side 0 = "left" (R), 1 = "right" (S).
 * Borrows the buffer (host or device memory) until spj_finish, as the
 * reference aliases it (src/query.cc:305-310). */
int spj_load_column(spj_handle_t *h, const void *tuples, int64_t num_tuples, int side);

/* void PrepareJoin(join_design_t), include/join_internals.hpp:320: validates the
 * design and allocates the device buffers of the plan. */
int spj_prepare(spj_handle_t *h, const spj_design_t *design);

/* void StartJoin(join_design_t), include/join_internals.hpp:321: enqueues the
 * column copies and the join on the instance's stream and returns. Columns
 * loaded since the last spj_prepare are prepared for first (with the current
 * design). */
int spj_start(spj_handle_t *h, const spj_design_t *design);

typedef struct {
    const spj_kv_pair_t *pairs;   /* host memory owned by the instance; valid until the
                                     next spj_start or spj_destroy */
    int64_t n_pairs;
    int num_rank;                 /* per-rank framing of ResultBuffers_t */
    const int64_t *rank_offsets;  /* num_rank + 1 pair offsets into `pairs` */
} spj_result_t;

/* ResultBuffers_t FinishJoin(), include/join_internals.hpp:322: waits for the join
 * and copies the pairs to host memory. No (0,0) padding is emitted. */
int spj_finish(spj_handle_t *h, spj_result_t *out);

/* Phase timings of the last join (CUDA events), milliseconds. */
typedef struct {
    double h2d_ms, partition_ms, join_ms, finish_ms, d2h_ms, total_ms;
    int64_t n_pairs;
    int64_t units;           /* work units executed */
    int64_t heavy_keys;      /* heavy keys of the join (found in the sample of S) */
    int64_t heavy_tuples;    /* pairs the first scatter pass emitted for heavy-key S tuples */
    int64_t max_r_partition; /* largest R partition */
    int64_t max_s_partition; /* largest S partition */
    int radix_bits;
    int table_slots;
    int join_alg;            /* the local-join algorithm the plan runs (enum spj_join_alg) */
} spj_stats_t;

/* void RecordLogs(struct timespec start, int rank_group), include/join_internals.hpp:323:
 * fills `out` and, when `print` is non-zero, writes one line per phase to stdout. */
int spj_record_logs(spj_handle_t *h, spj_stats_t *out, int print);

void spj_destroy(spj_handle_t *h);

/* ---------------------------------------------------- device-resident plan -- */
/* The B200 form of the reference's query plan (include/execution.hpp:15-157):
 * allocation happens once in spj_plan_create; spj_plan_execute allocates
 * nothing, never synchronises with the host and can be captured in a CUDA graph. */

typedef struct spj_plan spj_plan_t;

/* |R| and |S| below 2^32 - 2^24 - 1 tuples (output positions are 32-bit). */
int spj_plan_create(int64_t n_r, int64_t n_s, const spj_design_t *design, spj_plan_t **out);

/* Output capacity (pairs) that `out` must provide for this plan. */
int64_t spj_plan_output_capacity(const spj_plan_t *plan);

/* The planner's choice for one join: what spj_plan_create (batch_tuples = 0)
 * or spj_batch_create (batch_tuples = the batch's total |R| + |S|, its size
 * class's tuning applied) would run, computed from the device limits given
 * here instead of queried. It needs no device, so a caller can inspect a plan
 * anywhere (the EXPLAIN of this path). num_sms: 148 on B200;
 * max_smem_per_block: the opt-in shared memory per block, 232448 bytes on
 * B200. */
typedef struct {
    int32_t join_alg;           /* spj_join_alg the join runs (NPHJ replaces a hash join alone with |R| <= 2^22) */
    int32_t radix_bits;         /* partitions = 2^radix_bits (0: the non-partitioned join) */
    int32_t scatter_passes;     /* passes of the partitioning scatter: 1 or 2 (0: non-partitioned) */
    int32_t table_slots;        /* shared-memory table slots of a work unit (partitioned joins) */
    int64_t global_table_slots; /* the non-partitioned join's table in HBM (else 0) */
    int32_t heavy_sample;       /* S keys sampled for heavy keys joined on the fly (0: none) */
    int32_t unit_tuples;        /* S tuples per work unit */
    int32_t out_chunk;          /* output pairs a warp reserves at a time */
    int32_t chunk_tuples;       /* tuples per first-pass chunk */
} spj_plan_shape_t;

int spj_plan_describe(int64_t n_r, int64_t n_s, const spj_design_t *design, int num_sms, int max_smem_per_block,
                      int64_t batch_tuples, spj_plan_shape_t *out);

/* r, s, out: device pointers. n_out: device int64 that receives the pair count.
 * stream: a cudaStream_t (NULL = legacy default stream). */
int spj_plan_execute(spj_plan_t *plan, const spj_kv_pair_t *r, const spj_kv_pair_t *s, spj_kv_pair_t *out,
                     int64_t *n_out, void *stream);

/* Statistics of the last execution (synchronises with its stream). */
int spj_plan_stats(spj_plan_t *plan, spj_stats_t *out);

/* Per-kernel device times of one execution, from CUDA events recorded between
 * the launches on the execution's stream (milliseconds). */
typedef struct {
    double hist_ms;     /* partition histograms of R and S */
    double scan_ms;     /* offsets and partition starts */
    double scatter_ms;  /* radix scatter of R and S */
    double units_ms;    /* work-unit construction */
    double join_ms;     /* build + probe kernel */
    double fixup_ms;    /* output compaction */
    double total_ms;
} spj_kernel_times_t;

/* Times of the execution `back` runs ago (0 = last); the plan keeps the last 128. */
int spj_plan_kernel_times(spj_plan_t *plan, int back, spj_kernel_times_t *out);

void spj_plan_destroy(spj_plan_t *plan);

/* -------------------------------------------------------------- autotuning --
 * A per-size-class tuning table that the planner applies to the knobs a design
 * leaves at 0 (automatic) for the joins of a batch (a plan of two or more joins,
 * including the server's batches); a join planned alone keeps the planner's
 * choice. No counterpart in the reference, whose partition counts follow fixed
 * formulas.
 * A class is (floor(log2 |R|), floor(log2(|S| / |R|)) clamped to [0, 6]);
 * radix_bits_delta offsets the planner's fan-out (and so the pass count: one
 * scatter pass up to 2^8 partitions, two above), table_slots and unit_tuples
 * replace its choices when non-zero, and join_alg (spj_join_alg + 1; 0 = the
 * design's) picks the class's local-join algorithm among those with the
 * design's output semantics: the hash joins PHJ and NPHJ, or sort-merge and
 * nested loop. One batch may so mix algorithms. The table is filled by the
 * autotuner (spidjoin.autotune, which times candidates per class on the device)
 * and is process-wide; spj_tuning_set replaces it (n = 0 clears it). */
typedef struct {
    int log2_r, log2_ratio;
    int radix_bits_delta; /* -4..4 */
    int table_slots;      /* 0 = planner */
    int unit_tuples;      /* 0 = planner */
    int join_alg;         /* 0 = the design's; else spj_join_alg + 1 */
    int reserved[2];
} spj_tuning_t;
int spj_tuning_set(const spj_tuning_t *entries, int n);
/* Copies up to `capacity` entries; returns the table's size. */
int spj_tuning_get(spj_tuning_t *entries, int capacity);

/* ------------------------------------------------------------------ batches --
 * Many joins of uneven sizes and skew in one launch sequence: the kernels of a
 * batch plan cover every join, and one persistent work queue of
 * (join, partition, S range) units feeds the local-join CTAs. The plan's
 * tuning (fan-out, pass count, table size, output chunk) is chosen per join from
 * its sizes. No counterpart in the reference, which runs one JoinInstance per
 * join. Usage: create, bind the device pointers once, then execute any number
 * of times (execute allocates nothing, does not synchronise and can be captured
 * in a CUDA graph). Join j's pair count is written to n_out[j] (device array). */
int spj_batch_create(int n_joins, const int64_t *n_r, const int64_t *n_s, const spj_design_t *design,
                     spj_plan_t **out);
int64_t spj_batch_output_capacity(const spj_plan_t *plan, int join);
/* r, s, out: host arrays of n_joins device pointers; n_out: device int64[n_joins] (may be NULL). */
int spj_batch_bind(spj_plan_t *plan, const spj_kv_pair_t *const *r, const spj_kv_pair_t *const *s,
                   spj_kv_pair_t *const *out, int64_t *n_out);
int spj_batch_execute(spj_plan_t *plan, void *stream);
/* Counters of join `join` after an execution (synchronises). */
int spj_batch_stats(spj_plan_t *plan, int join, spj_stats_t *out);

/* ------------------------------------------------------------ join server --
 * A served stream of joins on one GPU with continuous batching. No counterpart
 * in the reference, which runs one JoinInstance per join. A worker thread
 * inside the server admits submitted joins in arrival order while their HBM
 * footprint (columns + output + partition scratch, estimated at 16 bytes per
 * input tuple) fits `hbm_budget_bytes`, forms one batch plan from everything
 * admitted at that moment (at most `max_batch` joins) and launches it on one of
 * `streams` streams, so batches overlap on the device. Scratch comes from a
 * private stream-ordered memory pool; submit and the worker never synchronise
 * the device. A join larger than the whole budget runs alone. Columns, output
 * and count stay owned by the caller and must stay valid and unchanged until
 * spj_server_wait returns for that id. Results equal those of the same join run
 * alone through spj_plan_execute (as pair multisets). */
typedef struct spj_server spj_server_t;
typedef struct {
    int64_t submitted, completed, failed, batches;
    int32_t max_inflight_batches, reserved0;
    double mean_batch;             /* joins per batch */
    uint64_t hbm_peak_bytes;       /* the most that admission held at once */
    uint64_t hbm_budget_bytes;
    double p50_ms, p99_ms, max_ms; /* submit -> completion latency */
} spj_server_stats_t;

int spj_server_create(const spj_design_t *design, uint64_t hbm_budget_bytes, int max_batch, int streams,
                      spj_server_t **out);
/* Output capacity (pairs) a join of these sizes must be given. */
int64_t spj_server_output_capacity(spj_server_t *server, int64_t n_r, int64_t n_s);
/* r, s: device columns (16-byte aligned); out: device pairs (16-byte aligned);
 * n_out: device int64 receiving the pair count; *id receives the request id. */
int spj_server_submit(spj_server_t *server, const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s,
                      int64_t n_s, spj_kv_pair_t *out, int64_t out_capacity, int64_t *n_out, int64_t *id);
/* Waits for request `id` (timeout_ms < 0: no limit; on timeout returns
 * SPJ_E_TIMEOUT and the id stays valid). On return the join's output and count
 * are in device memory; latency_ms (may be NULL) receives submit -> completion. */
int spj_server_wait(spj_server_t *server, int64_t id, double timeout_ms, double *latency_ms);
int spj_server_stats(spj_server_t *server, spj_server_stats_t *out);
/* hold != 0 pauses admission (submitted joins wait in the queue); hold = 0
 * resumes it, and everything queued that fits is admitted as one batch. Lets a
 * client hand over a group of joins that should run together. */
int spj_server_hold(spj_server_t *server, int hold);
/* Clears latencies and counters (e.g. after a warm-up phase). */
int spj_server_reset_stats(spj_server_t *server);
/* Finishes every queued and running join, then releases the server. */
void spj_server_destroy(spj_server_t *server);

/* The join for callers that cannot allocate device memory while they run it: a
 * database engine or other host runtime whose own pool allocator owns the whole
 * GPU (a cudaMalloc from inside a query would fail or take memory from that
 * pool), or a latency-bound loop that must not stall on the allocator
 * (cudaMalloc and cudaFree can synchronise the device). No counterpart in the
 * reference, whose host buffers are allocated per join. It computes what spj_plan_execute computes (the
 * partitioned hash join, SPJ_ALG_PHJ) but takes all scratch memory from one
 * fixed 32 MiB region inside the library, allocated once when the library loads
 * on a GPU and held until the process exits; the call allocates nothing.
 * Limits: |R| <= 2^20 and |S| <= 2^21 (larger sizes return SPJ_E_ARG);
 * out_capacity >= |S| + 2^21 pairs. r, s: device columns (16-byte aligned);
 * out: device pairs; n_out: device int64 that receives the pair count, or a
 * negative value if the join hit an internal capacity limit.
 * The first call on a device looks up the region's address and sets kernel
 * attributes; make that first call before capturing any stream. All calls share
 * the one region (the last call's contents stay in it): calls whose executions
 * overlap on the GPU -- on different streams or threads -- race and must be
 * serialised by the caller. */
int spj_join_noalloc(const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s, int64_t n_s, spj_kv_pair_t *out,
                     int64_t out_capacity, int64_t *n_out, void *stream);

/* Selection (src/dpu/include/select.h): out (device, capacity n) receives the
 * tuples of in[0, n) that pass `pred`, n_out (device int64) their count. The
 * tuples of each block of the input keep their order; the blocks' order in the
 * output is unspecified (a join consumes the result as a multiset). */
int spj_select(const spj_kv_pair_t *in, int64_t n, const spj_predicate_t *pred, spj_kv_pair_t *out, int64_t *n_out,
               void *stream);

/* The split before the rank-to-rank exchange of a join sharded over `world`
 * GPUs (this rank is `me`): the B200 form of the reference's global partition
 * scatter into per-rank packets ahead of its rotate-and-stream shuffle
 * (src/dpu/src/join/glb_partition_packet.c:420-464, src/queryHostFunc.cc:481-777).
 * The destination of a tuple is (glb_partition_hash(key) * world) >> 32, except
 * for heavy keys (heavy_keys: device uint32[n_heavy], n_heavy <= 256, sorted
 * ascending -- a caller precondition: the kernels binary-search the list, so an
 * unsorted one routes heavy tuples as ordinary ones),
 * SPID-Join's skew handling across ranks: with heavy_mode 1 (for S) a heavy
 * key's tuples stay on `me`; with heavy_mode 2 (for R, whose heavy tuples the
 * caller replicates to every rank) they leave the exchange; heavy_mode 0
 * ignores the list. Padding (key 0) is dropped.
 *
 * spj_exchange_split: out (device, n pairs) receives the routed tuples grouped
 * by destination: destination d's are out[off_d, off_d + counts[d]) with off the
 * exclusive prefix of counts (the order inside a group is unspecified);
 * counts: device int64[2 * world], the first `world` entries receive the group
 * sizes, the rest is workspace. Then an all-to-all moves the groups.
 *
 * spj_exchange_count + spj_exchange_scatter: the split fused into the send.
 * spj_exchange_count gives the per-destination sizes (counts: device
 * int64[world]); once every rank knows the size matrix, spj_exchange_scatter
 * writes each routed tuple straight into its destination's receive buffer.
 * dest_bufs: device array of `world` pointers to the ranks' receive buffers
 * (peer memory mapped into this process, e.g. symmetric memory, written over
 * NVLink); dest_offsets: device int64[world], where this rank's segment starts
 * in each destination buffer; cursor: device int64[world] workspace. The caller
 * orders the receivers' reads after every sender's kernel (a cross-GPU
 * barrier).
 *
 * All three allocate nothing and do not synchronise. */
int spj_exchange_split(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                       int n_heavy, int heavy_mode, spj_kv_pair_t *out, int64_t *counts, void *stream);
int spj_exchange_count(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                       int n_heavy, int heavy_mode, int64_t *counts, void *stream);
int spj_exchange_scatter(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                         int n_heavy, int heavy_mode, spj_kv_pair_t *const *dest_bufs, const int64_t *dest_offsets,
                         int64_t *cursor, void *stream);

/* -------------------------------------------------- sharded join (NCCL) ---- */
/* The join sharded over the GPUs of one node, one process per GPU, driven from
 * C: the B200 form of the reference's multi-rank join (src/queryHostFunc.cc:
 * 481-777, the rotate-and-stream shuffle; rank sets for skew,
 * glb_partition_count.c:317-318). Every rank owns a shard of R and of S. A call
 * (collective: every rank calls it, in the same order) finds the heavy keys of S
 * from a sample of every rank (a key whose estimated count reaches
 * heavy_share * |S_total| / world, at most 256 keys), all-gathers the R tuples
 * of those keys, sends every other tuple to rank (glb_partition_hash(key) *
 * world) >> 32 over NCCL (spj_exchange_split + grouped send/receive), and joins
 * what the rank received with a local plan. The union of the ranks' outputs is
 * the join of the whole relations.
 *
 * NCCL (libnccl.so.2) is loaded at the first call that needs it; without it
 * these return SPJ_E_UNSUPPORTED.
 *
 * spj_dist_unique_id: one rank makes the id (128 bytes) and hands it to the
 * others (any side channel). spj_dist_create: collective; binds the calling
 * thread's current CUDA device. spj_dist_set_heavy: mode 0 = no heavy keys,
 * 1 = heavy keys with more than one rank (default), 2 = always; share (default
 * 0.25) and sample (S keys a rank samples, default 65536) as above; every rank
 * sets the same values. spj_dist_join: r, s device shards (16-byte aligned);
 * *pairs receives a device pointer to this rank's *n_pairs output pairs, owned by
 * the handle and valid until its next join or its destruction; synchronises with
 * `stream`. spj_dist_heavy_keys: the heavy keys of the last join (returns their
 * number, copies at most `capacity` of them).
 *
 * Failures: a call that fails on one rank returns there, while the other ranks
 * may already wait in a collective of the same call, and NCCL has no timeout of
 * its own. spj_dist_abort (from any thread, e.g. a watchdog that learns of the
 * failure) aborts the rank's communicator: its pending collectives end with an
 * error, later joins return SPJ_E_STATE, and the handle can only be destroyed. */
typedef struct spj_dist spj_dist_t;
int spj_dist_unique_id(void *id_out);
int spj_dist_create(const void *unique_id, int world, int rank, const spj_design_t *design, spj_dist_t **out);
int spj_dist_set_heavy(spj_dist_t *d, int mode, double heavy_share, int sample);
int spj_dist_join(spj_dist_t *d, const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s, int64_t n_s,
                  const spj_kv_pair_t **pairs, int64_t *n_pairs, void *stream);
int spj_dist_heavy_keys(const spj_dist_t *d, uint32_t *keys, int capacity);
int spj_dist_abort(spj_dist_t *d);
void spj_dist_destroy(spj_dist_t *d);

/* Histogram of glb_partition_hash(key) & (2^bits - 1) over a device column (key-0
 * tuples skipped): the B200 form of the global partition count kernel
 * (src/dpu/src/join/glb_partition_count.c:119-371, partition_type 0). hist is a
 * device array of 2^bits uint32 counters. */
int spj_partition_histogram(const spj_kv_pair_t *tuples, int64_t n, int bits, uint32_t *hist, void *stream);

/* Order-independent checksum of a device pair array: the wrapping sum of
 * splitmix64((u64)lvalue << 32 | rvalue). */
int spj_checksum_device(const spj_kv_pair_t *pairs, const int64_t *n_dev, uint64_t *sum_dev, void *stream);

/* -------------------------------------------------- synthetic relations ---- */
/* The seeded generator of the benchmark relations (the reference's driver,
 * test/join/main.cc:30-48, leaves Zipf inputs to external files): R keys are a
 * permutation of 1..n_r with payload = row id; S payload = row id and S keys are
 * R keys drawn uniformly (zipf_s = 0) or Zipf(zipf_s) over a seeded rank order.
 * expected_checksum receives the checksum of the exact join output. */
int spj_generate_host(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r,
                      spj_kv_pair_t *s, uint64_t *expected_checksum, int nthreads);
int spj_generate_device(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r,
                        spj_kv_pair_t *s, uint64_t *expected_checksum_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SPIDJOIN_H */
