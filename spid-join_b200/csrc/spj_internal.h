// spj_internal.h -- plan layout shared by the kernels and the host orchestration.
//
// A plan describes a batch of J joins (J = 1 for the plain join). Every kernel
// covers all joins of the batch in one launch: chunks, partitions and coarse
// buckets of all relations live in flat index spaces, mapped back to
// (relation, local index) through prefix arrays, and the join kernels pull
// (join, partition, S range) work units from one queue.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/spidjoin.h"
#include "spj_common.h"

namespace spj {

constexpr int kHistThreads = 1024;
constexpr int kScatterThreads = 512;
constexpr int kScatterBlocksPerSM = 2;  // resident scatter CTAs per SM (shared memory and registers)
constexpr int kJoinThreads = 1024;
// Relation sizes stay below this, so output positions (|S| + output slack) fit 32 bits.
constexpr long long kMaxTuples = 0xFFFFFFFFll - (1ll << 24);
constexpr int kOutChunk = 1024;       // output pairs reserved per warp at a time
constexpr int kMaxHoles = 12288;      // per join: warps of the emitting kernels (one hole each)
constexpr int kUpSlots = kMaxHoles + 2;  // chunks that the output's tail [N, reserved) can span
constexpr int kMaxRadixBits = 15;
constexpr int kMaxPassBits = 8;       // buckets per scatter pass <= 256
constexpr int kTile = 4096;           // tuples sorted per tile in shared memory
constexpr int kDefaultTableSlots = 12288;  // 96 KB of shared memory
constexpr int kDefaultUnitTuples = 65536;
// Heavy keys of one join (S keys frequent enough in a sample of S to be joined on
// the fly during the first scatter pass instead of being partitioned).
constexpr int kHeavySlots = 512;          // open-addressing slots of the heavy table
constexpr int kHeavyMax = 256;            // heavy keys per join (load <= 1/2)
constexpr int kHeavySampleDefault = 16384;  // a key of 1/1000 of S is seen ~16 times
constexpr int kHeavySampleMax = 1 << 20;
constexpr int kSampleSlots = 16384;       // shared-memory counting table of the sample
constexpr double kHeavyMinShare = 0.6;    // automatic mode: least sample share of the heavy keys
// Shared-memory hash-table slots (8 bytes each) a join CTA can hold on a device
// with `max_smem` bytes of opt-in shared memory per block, leaving room for the
// join kernels' static shared memory; pairs of slots are probed together.
inline int max_table_slots_for(int max_smem) { return ((max_smem - 12288) / 8) & ~1; }

// One relation (R or S) of one join.
struct RelDev {
    const Tuple *in;     // input column (device)
    Tuple *out;          // partitioned column
    Tuple *tmp;          // pass-1 (coarse) layout when two passes are used
    uint32_t n;          // tuples
    uint32_t chunk;      // tuples per chunk (even)
    uint32_t nchunks;
    uint32_t join;       // owning join
    uint32_t *hist;      // [nchunks][F] counts, then exclusive offsets within each partition
    uint32_t *chist;     // [nchunks][F1] counts of the coarse buckets (two-pass scatter)
    uint32_t *total;     // [F] tuples per partition
    uint32_t *base;      // [F] partition starts
    Pred pred;           // selection ahead of the join (field 0: none)
};

// The heavy table of one join: written by the sampling kernel (keys), completed
// by the count pass over R (the payload of one R tuple per heavy key, `found`),
// read by the first scatter pass over S. Key 0 marks an empty slot.
struct HeavyTab {
    uint32_t n;        // heavy keys
    uint32_t pad[3];
    uint32_t key[kHeavySlots];
    uint32_t pay[kHeavySlots];
    uint32_t found[kHeavySlots];
};

struct Hole {
    unsigned long long begin, end;
};

// Per-join counters of one execution (zeroed at its start).
struct JoinCtr {
    unsigned long long out_reserved;  // output slots handed out (pairs + holes)
    unsigned long long n_out;         // final pair count
    unsigned long long gap_total;     // fix-up: hole space below n_out
    unsigned int hole_count;
    unsigned int error;               // 1 table, 2 output, 4 work list, 8 holes, 16 fix-up, 32 timeout
    unsigned int max_r_part, max_s_part;
    unsigned int n_gaps, n_data;
    unsigned int units;               // work units of the join
    unsigned int unit_base;           // its first unit in the queue
    unsigned int unit_fill;
    unsigned int heavy_keys;          // keys joined on the fly
    unsigned long long heavy_tuples;  // S tuples joined on the fly (pairs emitted by the scatter)
    unsigned int probe_done;          // direct non-partitioned probe: CTAs finished
};

// Per-join constants and output state.
struct JoinDev {
    int bits;             // radix bits of the partition fan-out
    int fine_bits;        // bits resolved by the second scatter pass (0 = one pass)
    int table_slots;      // shared-memory table entries (8 bytes each)
    int alg;              // spj_join_alg
    int skew_mode;
    int group;            // rank_set * bank_set
    int keep_unmatched;   // SMJ/NL rewrite S in place and keep unmatched tuples
    uint32_t unit_tuples;
    uint32_t item_target; // tuples per pass-2 work item
    uint32_t out_chunk;   // output pairs a warp reserves at a time (<= kOutChunk)
    Tuple *out;
    unsigned long long out_cap;
    unsigned long long *n_out_user;   // optional device destination of the pair count
    JoinCtr *ctr;
    Hole *holes, *gaps, *datas;
    unsigned long long *gap_off, *data_off;
    unsigned long long *gtable;       // non-partitioned hash join: global table
    unsigned long long gtable_slots;
    HeavyTab *heavy;                  // null: no heavy-key path for this join
    uint32_t heavy_sample;            // S keys sampled to find heavy keys
    int heavy_auto;                   // the planner chose the sample: keep heavy keys only when
                                      // they hold at least kHeavyMinShare of it
};

// A work unit: join j, partition p, S range [s_begin, s_end) of the partitioned S column.
struct Unit {
    uint32_t p;
    uint32_t s_begin;
    uint32_t s_end;
    uint32_t join;
};

// Batch-wide queues (zeroed per execution).
// The unit queue holds each local-join algorithm's units in one contiguous
// range, [alg_begin[a], alg_begin[a + 1]), so every join kernel of a batch whose
// joins use different algorithms claims only its own.
struct BatchCtr {
    unsigned int unit_count, unit_next;
    unsigned int item_count, item_next;
    unsigned int error;
    unsigned int alg_begin[5];
    unsigned int alg_next[4];
};

// Kernel-parameter view of a plan.
struct PlanDev {
    RelDev *rel;              // [2J]: rel[2j] = R of join j, rel[2j+1] = S of join j
    JoinDev *join;            // [J]
    uint32_t *chunk_prefix;   // [2J+1] first flat chunk of each relation
    uint32_t *part_prefix;    // [2J+1] first flat partition of each relation (F_j each)
    uint32_t *coarse_prefix;  // [2J+1] first flat coarse bucket (F1_j, or 0 for one pass)
    uint32_t *jpart_prefix;   // [J+1] first flat partition of each join (R side)
    uint32_t nrel, njoin;
    uint32_t total_chunks, total_parts, total_coarse, total_jparts;
    int max_bits;             // histogram shared memory
    int max_table_slots;      // join-kernel shared memory
    int alg_mask;             // 1 << spj_join_alg of every algorithm some join uses
    int any_two_pass;
    int any_heavy;            // some join samples heavy keys
    Unit *units;
    uint32_t max_units;
    uint4 *items;             // pass-2 work items: (relation, coarse bucket, first chunk, end chunk)
    uint32_t max_items;
    BatchCtr *bctr;
    JoinCtr *jctr;            // [J], contiguous after bctr (one memset clears both)
};

// Host-side description of one join of a plan.
struct JoinHost {
    int64_t n_r = 0, n_s = 0;
    JoinDev dev{};
    RelDev rel[2]{};
};

// Per-join tuning chosen from the sizes and the design.
struct JoinShape {
    int bits = 0, fine_bits = 0, table_slots = 0;
    uint32_t nchunks[2] = {1, 1}, chunk[2] = {2, 2};
    uint32_t item_target = 0;
    uint32_t out_chunk = kOutChunk;
    uint32_t unit_tuples = kDefaultUnitTuples;
    unsigned long long gtable_slots = 0;
    uint32_t heavy_sample = 0;  // 0: no heavy-key path
    int heavy_auto = 0;
    int alg = SPJ_ALG_PHJ;      // the join's local-join algorithm
};

}  // namespace spj

struct spj_plan {
    int64_t n_r = 0, n_s = 0;      // join 0 (plain plans)
    spj_design_t design{};
    std::vector<spj::JoinHost> joins;
    std::vector<spj::JoinShape> shapes;
    spj::PlanDev dev{};
    int device = 0;
    int num_sms = 0;
    int join_blocks = 0;
    void *arena = nullptr;         // one device allocation for all scratch
    size_t arena_bytes = 0;
    size_t desc_offset = 0;        // descriptor arrays inside the arena
    std::vector<unsigned char> desc_host;  // their host image
    static constexpr int kRing = 128;   // executions whose kernel times are kept
    static constexpr int kMarks = 7;    // events per execution
    cudaEvent_t ring[kRing][kMarks]{};
    int ring_next = 0;                  // slot of the next execution
    int ring_filled = 0;
    bool have_events = false;
    std::string last_error;
};

namespace spj {
int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);

// batch_tuples: all tuples of the plan's joins when the join is one of many (0 alone)
// tune: the autotuner's entry for this size class, or null
JoinShape plan_shape(int64_t n_r, int64_t n_s, const spj_design_t &d, int sms, int max_slots, bool alone,
                     int64_t batch_tuples, const spj_tuning_t *tune);
const spj_tuning_t *find_tuning(int64_t n_r, int64_t n_s, spj_tuning_t *out);
// Computes the arena layout of pl->joins/pl->shapes (arena == nullptr: size only)
// and fills pl->dev, the per-join descriptors and the host image of the
// descriptor arrays.
size_t layout_plan(spj_plan *pl, char *arena, bool image);
// keep_r (one-join plans): R's partitions from the plan's previous execution on
// the same stream are reused; only S is counted and scattered.
cudaError_t launch_pipeline(spj_plan *pl, cudaStream_t st, bool keep_r = false);
cudaError_t init_single(spj_plan *pl, cudaStream_t st, bool keep_r = false);
// spj_plan_execute with keep_r (see launch_pipeline).
int plan_execute(spj_plan *pl, const spj_kv_pair_t *r, const spj_kv_pair_t *s, spj_kv_pair_t *out, int64_t *n_out,
                 cudaStream_t st, bool keep_r);
// alg_mask: 1 << spj_join_alg of each algorithm the plan's joins use; the CTAs
// per SM that every one of those join kernels can keep resident.
cudaError_t configure_kernels(int table_slots, int alg_mask, int *join_blocks_per_sm);
int create_plan_stream(int J, const int64_t *n_r, const int64_t *n_s, const spj_design_t *design,
                       const spj_kv_pair_t *const *r, const spj_kv_pair_t *const *s, spj_kv_pair_t *const *out,
                       int64_t *const *n_out, cudaMemPool_t pool, cudaStream_t st, spj_plan_t **pout,
                       size_t *bytes);
void destroy_plan_stream(spj_plan_t *pl, cudaStream_t st);
int64_t join_output_capacity(int64_t n_r, int64_t n_s, const spj_design_t &d, bool alone);
int join_ctr_status(unsigned err, unsigned max_r_part);
}  // namespace spj
