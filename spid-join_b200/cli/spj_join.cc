// spj_join -- command-line driver of the join, with the knobs of the
// reference's driver (test/join/main.cc:73-118):
//   -s input_size (|R|)  -r rank_num  -z zipf_factor (Zipf exponent x 100)
//   -t rs_ratio (|S|/|R|)  -R rank_set  -B bank_set
// plus -a algorithm (phj|nphj|smj|nl), -n repetitions, -S seed, -o (result
// buffers owned by the caller), -P (the reference's padded per-rank layout of
// 64 DPU blocks; implies -o) and -E (print the plan the join would run, from
// spj_plan_describe with the B200's limits, and exit without touching a GPU).
// -h, -p and -f take an argument and are ignored, as in the reference.
//
// With -z 0 the relations are the reference driver's (test/join/main.cc:33-43):
// R[i] = (i+1, i+3) and S[i] = (i/ratio + 1, i/ratio + 3). With -z > 0 the
// reference reads pre-generated files; here S keys are drawn Zipf(z/100) over
// a seeded shuffle of R's keys by spj_generate_host. The output is checked by
// count and by the order-independent 64-bit checksum (with -P over the non-(0,0)
// pairs, which needs an output without a (0,0) pair of its own, as -z 0's is);
// the exit status is 0 when it matches, 1 when it does not and 2 on an error.
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <string>
#include <vector>

#include "pidjoin.hpp"

using namespace pidjoin;

// the output checksum's digest: the splitmix64 finaliser of (lvalue << 32 | rvalue)
static uint64_t splitmix64(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static uint64_t pair_sum(const kv_pair_t *p, int64_t n, bool skip_zero, int64_t *counted) {
    uint64_t s = 0;
    int64_t c = 0;
    for (int64_t i = 0; i < n; i++) {
        if (skip_zero && p[i].lvalue == 0 && p[i].rvalue == 0) continue;  // block padding
        s += splitmix64((uint64_t)p[i].lvalue << 32 | p[i].rvalue);
        c++;
    }
    *counted = c;
    return s;
}

int main(int argc, char **argv) {
    join_design_t d;
    d.primary_key = "order";
    d.foreign_key = "l";
    std::string alg = "phj";
    int reps = 1;
    bool owned = false;  // -o: result buffers owned by the caller, as the reference hands them out
    bool padded = false; // -P: the reference's transfer layout, 64 zero-padded DPU blocks per rank
    bool explain = false; // -E: the plan only
    uint64_t seed = 0x5EED5EEDull;
    if (argc < 2) {
        fprintf(stderr, "usage: %s -s |R| [-r ranks] [-z zipf*100] [-t |S|/|R|] [-R rank_set] [-B bank_set] "
                        "[-a phj|nphj|smj|nl] [-n reps] [-S seed] [-o] [-P] [-E]\n", argv[0]);
        return 0;
    }
    int opt;
    while ((opt = getopt(argc, argv, "s:r:z:t:R:B:h:p:f:a:n:S:oPE")) != -1) {
        switch (opt) {
            case 's': d.input_size = atoll(optarg); break;
            case 'r': d.rank_num = atoi(optarg); break;
            case 'z': d.zipf_factor = atoi(optarg); break;
            case 't': d.rs_ratio = atoi(optarg); break;
            case 'R': d.rank_set = atoi(optarg); break;
            case 'B': d.bank_set = atoi(optarg); break;
            case 'a': alg = optarg; break;
            case 'n': reps = atoi(optarg); break;
            case 'S': seed = strtoull(optarg, nullptr, 0); break;
            case 'o': owned = true; break;
            case 'P': padded = owned = true; break;
            case 'E': explain = true; break;
            default: break;
        }
    }
    if (alg == "phj") d.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_PHJ;
    else if (alg == "nphj") d.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_NPHJ;
    else if (alg == "smj") d.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_SMJ;
    else if (alg == "nl") d.join_alg = JOIN_DESIGN_JOIN_ALGORITHM_NL;
    else {
        fprintf(stderr, "unknown algorithm %s\n", alg.c_str());
        return 2;
    }
    const int64_t n_r = d.input_size, n_s = d.input_size * (int64_t)d.rs_ratio;
    if (n_r <= 0 || d.rs_ratio <= 0 || d.rank_num <= 0 || d.rank_set <= 0 || d.rank_num % d.rank_set) {
        fprintf(stderr, "bad sizes or rank layout\n");
        return 2;
    }
    if (explain) {
        const spj_design_t c = d.to_c();
        spj_plan_shape_t sh;
        if (spj_plan_describe(n_r, n_s, &c, 148, 232448, 0, &sh) != SPJ_OK) {
            fprintf(stderr, "%s\n", spj_last_error());
            return 2;
        }
        static const char *const names[] = {"phj", "nphj", "smj", "nl"};
        printf("plan: |R|=%lld |S|=%lld alg=%s radix_bits=%d passes=%d table_slots=%d global_table_slots=%lld "
               "heavy_sample=%d unit_tuples=%d out_chunk=%d chunk_tuples=%d\n",
               (long long)n_r, (long long)n_s, names[sh.join_alg], sh.radix_bits, sh.scatter_passes, sh.table_slots,
               (long long)sh.global_table_slots, sh.heavy_sample, sh.unit_tuples, sh.out_chunk, sh.chunk_tuples);
        return 0;
    }
    std::vector<kv_pair_t> R(n_r), S(n_s);
    uint64_t expect = 0;
    if (d.zipf_factor == 0) {
        for (int64_t i = 0; i < n_r; i++) R[i] = {(uint32_t)(i + 1), (uint32_t)(i + 3)};
        for (int64_t i = 0; i < n_s; i++) {
            const uint32_t k = (uint32_t)(i / d.rs_ratio);
            S[i] = {k + 1, k + 3};
            expect += splitmix64((uint64_t)(k + 3) << 32 | (k + 3));
        }
    } else if (spj_generate_host(seed, n_r, n_s, d.zipf_factor / 100.0, R.data(), S.data(), &expect, 0) != SPJ_OK) {
        fprintf(stderr, "generator: %s\n", spj_last_error());
        return 2;
    }
    try {
        JoinInstance join_instance(d.rank_num, d.rank_set, d.rank_num / d.rank_set);
        join_instance.LoadColumn(R.data(), n_r, "left");
        join_instance.LoadColumn(S.data(), n_s, "right");
        join_instance.PrepareJoin(d);
        int bad = 0;
        for (int it = 0; it < reps; it++) {
            struct timespec start;
            clock_gettime(CLOCK_MONOTONIC, &start);
            join_instance.StartJoin(d);
            ResultBuffers_t res = join_instance.FinishJoin(owned, padded);
            join_instance.RecordLogs(start, 0);
            int64_t n = 0, bytes = 0;
            uint64_t sum = 0;
            for (size_t r = 0; r < res.first.size(); r++) {
                int64_t c = 0;
                sum += pair_sum(res.first[r], res.second[r] / 8, padded, &c);
                n += c;
                bytes += res.second[r];
            }
            if (padded) printf("padded layout: %lld bytes in %zu ranks of 64 blocks\n", (long long)bytes, res.first.size());
            const bool ok = n == n_s && sum == expect;
            printf("check: %s pairs=%lld expected=%lld checksum=%016llx expected=%016llx\n", ok ? "ok" : "MISMATCH",
                   (long long)n, (long long)n_s, (unsigned long long)sum, (unsigned long long)expect);
            bad += !ok;
            if (owned)
                for (auto *p : res.first) free(p);
        }
        return bad ? 1 : 0;
    } catch (const Error &e) {
        fprintf(stderr, "%s\n", e.what());
        return 2;
    }
}
