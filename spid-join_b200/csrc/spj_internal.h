// spj_internal.h -- plan layout shared by the kernels and the host orchestration.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/spidjoin.h"
#include "spj_common.h"

namespace spj {

constexpr int kHistThreads = 1024;
constexpr int kScatterThreads = 512;
constexpr int kJoinThreads = 1024;
constexpr int kOutChunk = 1024;      // output pairs reserved per warp at a time
constexpr int kMaxHoles = 12288;     // warps of the emitting kernels (one hole each)
constexpr int kHoleSortSlots = 16384; // power of two >= kMaxHoles
constexpr int kMaxRadixBits = 15;
constexpr int kMaxPassBits = 8;      // buckets per scatter pass <= 256
constexpr int kTile = 4096;          // tuples sorted per tile in shared memory
constexpr int kDefaultTableSlots = 12288;  // 96 KB of shared memory
constexpr int kDefaultUnitTuples = 65536;
constexpr int kHeavyCap = 1024;      // heavy keys joined on the fly

// One relation's partitioning state.
struct RelDev {
    const Tuple *in;     // input column (device)
    Tuple *out;          // partitioned column
    Tuple *tmp;          // pass-1 (coarse) layout when two passes are used
    uint32_t n;          // tuples
    uint32_t chunk;      // tuples per chunk (even)
    uint32_t nchunks;
    uint32_t *hist;      // [nchunks][F] counts, then exclusive offsets within each partition
    uint32_t *chist;     // [nchunks][F1] counts of the coarse buckets (two-pass scatter)
    uint32_t *total;     // [F] tuples per partition
    uint32_t *base;      // [F] partition starts
};

// A work unit: partition p, S range [s_begin, s_end) of the partitioned S column.
struct Unit {
    uint32_t p;
    uint32_t s_begin;
    uint32_t s_end;
    uint32_t pad;
};

struct Hole {
    unsigned long long begin, end;
};

// Device-side counters of one execution (zeroed at the start of each execution).
struct Counters {
    unsigned long long out_reserved;  // output slots handed out (pairs + holes)
    unsigned int unit_count;
    unsigned int unit_next;
    unsigned int hole_count;
    unsigned int error;               // bit 0: table overflow, bit 1: output overflow
    unsigned int max_r_part;
    unsigned int max_s_part;
    unsigned int heavy_keys;
    unsigned int pad;
    unsigned long long heavy_tuples;
    unsigned long long n_out;         // final pair count
    unsigned long long gap_total;     // fix-up: hole space below n_out
    unsigned int n_gaps, n_data;
    unsigned int item_count, item_next;  // pass-2 work list
};

struct JoinParams {
    int bits;             // radix bits of the partition fan-out
    int fine_bits;        // bits resolved by the second scatter pass (0 = one pass)
    int table_slots;      // shared-memory table entries (8 bytes each)
    int alg;              // spj_join_alg
    int skew_mode;
    int group;            // rank_set * bank_set
    uint32_t unit_tuples;
    int keep_unmatched;   // SMJ/NL rewrite S in place and keep unmatched tuples
};

struct PlanDev {
    RelDev rel[2];        // 0 = R, 1 = S
    Unit *units;
    uint32_t max_units;
    uint4 *items;         // pass-2 work items: (relation, coarse bucket, first chunk, end chunk)
    uint32_t max_items;
    Hole *holes;
    Hole *gaps;           // fix-up scratch
    Hole *datas;
    unsigned long long *gap_off;
    unsigned long long *data_off;
    Counters *ctr;
    Tuple *out;
    unsigned long long out_cap;
    unsigned long long *gtable;       // global table of the non-partitioned hash join
    unsigned long long *n_out_user;   // optional user destination of the pair count
};

}  // namespace spj

struct spj_plan {
    int64_t n_r = 0, n_s = 0;
    spj_design_t design{};
    spj::JoinParams jp{};
    spj::PlanDev dev{};
    int device = 0;
    int num_sms = 0;
    int join_blocks = 0;
    uint32_t item_target = 0;    // tuples per pass-2 work item
    uint64_t gtable_slots = 0;   // non-partitioned hash join: table slots (power of two)
    void *arena = nullptr;        // one device allocation for all scratch
    size_t arena_bytes = 0;
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
}  // namespace spj
