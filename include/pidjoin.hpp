// pidjoin.hpp -- C++ facade of libspidjoin with the reference's host API.
//
// The reference (yonsei-hpcp/spid-join) exposes its join as the C++ class
// pidjoin::JoinInstance (include/join_internals.hpp:280-324) configured by
// pidjoin::join_design_t (include/idpHandler.hpp:131-145), with kv_pair_t
// (include/type_defs.hpp:53-56) tuples and ResultBuffers_t
// (include/type_defs.hpp:82) results. This header keeps those names, argument
// meanings and call order over the C ABI in spidjoin.h, so a caller written
// against the reference (e.g. its driver test/join/main.cc) compiles against
// this header and links -lspidjoin. Differences: errors throw pidjoin::Error
// instead of exit(-1); result buffers hold exactly the join's pairs (no (0,0)
// padding) and are owned by the instance until the next StartJoin.
#ifndef PIDJOIN_HPP
#define PIDJOIN_HPP

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "spidjoin.h"

#define JOIN_DESIGN_JOIN_ALGORITHM_PHJ 0
#define JOIN_DESIGN_JOIN_ALGORITHM_NPHJ 1
#define JOIN_DESIGN_JOIN_ALGORITHM_SMJ 2
#define JOIN_DESIGN_JOIN_ALGORITHM_NL 3

namespace pidjoin {

typedef spj_kv_pair_t kv_pair_t;

// Per rank: the pair buffers and their sizes in bytes (include/type_defs.hpp:82).
typedef std::pair<std::vector<kv_pair_t *>, std::vector<int64_t>> ResultBuffers_t;

// include/idpHandler.hpp:131-145, same fields and defaults; the B200 tuning
// fields follow (0 = chosen by the planner).
struct join_design_t {
    int64_t input_size = 500000;
    int rank_num = 16;
    int zipf_factor = 0;  // Zipf exponent x 100
    int rs_ratio = 8;
    int rank_set = 1;
    int bank_set = 1;
    bool tpch_example = false;
    int join_alg = JOIN_DESIGN_JOIN_ALGORITHM_PHJ;
    std::string primary_key;
    std::string foreign_key;
    int identical_value_percent = 0;
    // B200 tuning
    int radix_bits = 0;
    int skew_mode = SPJ_SKEW_ADAPTIVE;
    int unit_tuples = 0;
    int heavy_sample = 0;
    int table_slots = 0;
    // selections on R and S ahead of the join (src/dpu/include/select.h predicates)
    spj_predicate_t select_r{SPJ_PRED_NONE, SPJ_PRED_EQ, 0u, 0u};
    spj_predicate_t select_s{SPJ_PRED_NONE, SPJ_PRED_EQ, 0u, 0u};

    spj_design_t to_c() const {
        spj_design_t d;
        spj_design_default(&d);
        d.input_size = input_size;
        d.rank_num = rank_num;
        d.zipf_factor = zipf_factor;
        d.rs_ratio = rs_ratio;
        d.rank_set = rank_set;
        d.bank_set = bank_set;
        d.tpch_example = tpch_example ? 1 : 0;
        d.join_alg = join_alg;
        d.radix_bits = radix_bits;
        d.skew_mode = skew_mode;
        d.unit_tuples = unit_tuples;
        d.heavy_sample = heavy_sample;
        d.table_slots = table_slots;
        d.select_r = select_r;
        d.select_s = select_s;
        return d;
    }
};

class Error : public std::runtime_error {
public:
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char *what) {
    if (rc != SPJ_OK) throw Error(rc, std::string(what) + ": " + spj_last_error());
}

class JoinInstance {
    spj_handle_t *h_ = nullptr;
    spj_result_t last_{};

public:
    int num_rank_allocated = 0;
    int num_rankgroup = 0;
    int num_rank_in_rankgroup = 0;

    // include/join_internals.hpp:304-306
    JoinInstance() : JoinInstance(1, 1, 1) {}
    explicit JoinInstance(int num_rank_allocated_) : JoinInstance(num_rank_allocated_, 1, num_rank_allocated_) {}
    JoinInstance(int num_rank_allocated_, int num_rankgroup_, int num_rank_in_rankgroup_)
        : num_rank_allocated(num_rank_allocated_),
          num_rankgroup(num_rankgroup_),
          num_rank_in_rankgroup(num_rank_in_rankgroup_) {
        check(spj_create(num_rank_allocated_, num_rankgroup_, num_rank_in_rankgroup_, &h_), "JoinInstance");
    }
    ~JoinInstance() { spj_destroy(h_); }
    JoinInstance(const JoinInstance &) = delete;
    JoinInstance &operator=(const JoinInstance &) = delete;

    // include/join_internals.hpp:316; "left" = R (build), "right" = S (probe).
    // The buffer is borrowed until FinishJoin, as in the reference.
    void LoadColumn(void *data_ptr, int64_t num_tuples, std::string col_name) {
        if (col_name != "left" && col_name != "right") throw Error(SPJ_E_ARG, "LoadColumn: col_name " + col_name);
        check(spj_load_column(h_, data_ptr, num_tuples, col_name == "right"), "LoadColumn");
    }

    // include/join_internals.hpp:317 (the reference accepts "phj" and "smj";
    // "nphj" and "nl" select the other two local joins).
    void ExecuteJoin(std::string join_type, join_design_t join_design) {
        if (join_type == "phj")
            join_design.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_PHJ;
        else if (join_type == "smj")
            join_design.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_SMJ;
        else if (join_type == "nphj")
            join_design.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_NPHJ;
        else if (join_type == "nl")
            join_design.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_NL;
        else
            throw Error(SPJ_E_ARG, "ExecuteJoin: not supported join algorithm " + join_type);
        PrepareJoin(join_design);
        StartJoin(join_design);
        FinishJoin();
    }

    void PrepareJoin(join_design_t join_design) {
        const spj_design_t d = join_design.to_c();
        check(spj_prepare(h_, &d), "PrepareJoin");
    }
    void StartJoin(join_design_t join_design) {
        const spj_design_t d = join_design.to_c();
        check(spj_start(h_, &d), "StartJoin");
    }

    // Per-rank pair buffers and their byte sizes. By default the buffers are
    // slices of host memory owned by the instance (valid until the next
    // StartJoin). With caller_owned, each rank's pairs are copied into its own
    // aligned_alloc'd buffer that the caller releases with free(), as the
    // reference hands out its result buffers (src/queryHostFunc.cc:1089).
    //
    // With dpu_blocks (implies caller_owned), each rank's buffer has the
    // reference's transfer layout instead (src/queryHostFunc.cc:1058-1126 over
    // the blocks src/dpu/src/join/finish_join.c:99-129 pads): 64 blocks of one
    // size, each holding its pairs followed by (0,0) padding, and the byte size
    // reported is that of the 64 padded blocks. The rank's pairs are dealt to
    // the blocks in order and evenly (block b takes pairs / 64 of them, one more
    // for the first pairs % 64 blocks; blocks hold ceil(pairs / 64)): this join
    // has no DPUs, so which pair lands in which block carries no meaning. As in
    // the reference, a (0,0) pair of the join itself cannot be told from padding.
    ResultBuffers_t FinishJoin(bool caller_owned = false, bool dpu_blocks = false) {
        check(spj_finish(h_, &last_), "FinishJoin");
        ResultBuffers_t out;
        for (int r = 0; r < last_.num_rank; r++) {
            const int64_t n = last_.rank_offsets[r + 1] - last_.rank_offsets[r];
            const int64_t bytes = 8 * n;
            kv_pair_t *src = const_cast<kv_pair_t *>(last_.pairs) + last_.rank_offsets[r];
            if (dpu_blocks) {
                constexpr int64_t kBlocks = 64;  // DPUs per rank (NUM_DPU_RANK)
                const int64_t per = (n + kBlocks - 1) / kBlocks;
                const int64_t padded = kBlocks * per * 8;
                kv_pair_t *dst = (kv_pair_t *)aligned_alloc(64, (size_t)((padded + 63) / 64 * 64 + 64));
                if (!dst) throw Error(SPJ_E_NOMEM, "FinishJoin: result buffer allocation failed");
                memset(dst, 0, (size_t)padded);
                const int64_t base = n / kBlocks, extra = n % kBlocks;
                for (int64_t b = 0, lo = 0; b < kBlocks; b++) {
                    const int64_t cnt = base + (b < extra ? 1 : 0);
                    if (cnt) memcpy(dst + b * per, src + lo, (size_t)cnt * 8);
                    lo += cnt;
                }
                out.first.push_back(dst);
                out.second.push_back(padded);
                continue;
            }
            if (caller_owned) {
                kv_pair_t *dst = (kv_pair_t *)aligned_alloc(64, (size_t)((bytes + 63) / 64 * 64 + 64));
                if (!dst) throw Error(SPJ_E_NOMEM, "FinishJoin: result buffer allocation failed");
                memcpy(dst, src, (size_t)bytes);
                src = dst;
            }
            out.first.push_back(src);
            out.second.push_back(bytes);
        }
        return out;
    }
    int64_t NumPairs() const { return last_.n_pairs; }

    // include/join_internals.hpp:323: prints the phase times of the last join
    // (CUDA events) and the wall time since `start`.
    void RecordLogs(struct timespec start, int rank_group) {
        spj_stats_t s;
        check(spj_record_logs(h_, &s, 1), "RecordLogs");
        struct timespec now;
        clock_gettime(CLOCK_MONOTONIC, &now);
        const double ms = (now.tv_sec - start.tv_sec) * 1e3 + (now.tv_nsec - start.tv_nsec) / 1e6;
        printf("rank_group %d: %lld pairs, %.3f ms since start\n", rank_group, (long long)s.n_pairs, ms);
    }
    spj_stats_t Stats() {
        spj_stats_t s;
        check(spj_record_logs(h_, &s, 0), "Stats");
        return s;
    }
};

}  // namespace pidjoin

#endif  // PIDJOIN_HPP
