// spj_dist_check -- the sharded join driven from C++ with no Python: one process
// per GPU, the NCCL id made by rank 0. Here a world of one rank (every rank
// would call the same sequence with its own shards): the seeded relations are
// generated on the device, joined by spj_dist_join, and the pairs checked by
// count and order-independent checksum against the generator's answer.
//   spj_dist_check [|R|] [|S|] [zipf]      exit status 0 when the result matches
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include "spidjoin.h"

#define CHECK(call)                                                         \
    do {                                                                    \
        int rc_ = (call);                                                   \
        if (rc_ != SPJ_OK) {                                                \
            fprintf(stderr, "%s: %d %s\n", #call, rc_, spj_last_error());   \
            return 2;                                                       \
        }                                                                   \
    } while (0)

int main(int argc, char **argv) {
    const int64_t n_r = argc > 1 ? atoll(argv[1]) : (1 << 18);
    const int64_t n_s = argc > 2 ? atoll(argv[2]) : (1 << 21);
    const double zipf = argc > 3 ? atof(argv[3]) : 1.5;
    spj_kv_pair_t *r = nullptr, *s = nullptr;
    uint64_t *expect = nullptr, *sum = nullptr;
    int64_t *n_dev = nullptr;
    if (cudaMalloc(&r, n_r * 8) || cudaMalloc(&s, n_s * 8) || cudaMalloc(&expect, 8) || cudaMalloc(&sum, 8) ||
        cudaMalloc(&n_dev, 8)) {
        fprintf(stderr, "cudaMalloc failed\n");
        return 2;
    }
    cudaMemset(expect, 0, 8);
    CHECK(spj_generate_device(0x5EED5EEDull, n_r, n_s, zipf, r, s, expect, nullptr));

    char id[128];
    CHECK(spj_dist_unique_id(id));  // rank 0 makes it; other ranks would receive it
    spj_design_t d;
    spj_design_default(&d);
    d.rank_num = 1;
    spj_dist_t *dj = nullptr;
    CHECK(spj_dist_create(id, 1, 0, &d, &dj));
    CHECK(spj_dist_set_heavy(dj, 2, 0.25, 1 << 16));  // heavy keys even with one rank
    int bad = 0;
    for (int it = 0; it < 2; it++) {
        const spj_kv_pair_t *pairs = nullptr;
        int64_t n = 0;
        CHECK(spj_dist_join(dj, r, n_r, s, n_s, &pairs, &n, nullptr));
        cudaMemcpy(n_dev, &n, 8, cudaMemcpyHostToDevice);
        cudaMemset(sum, 0, 8);
        CHECK(spj_checksum_device(pairs, n_dev, sum, nullptr));
        uint64_t got = 0, want = 0;
        cudaMemcpy(&got, sum, 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(&want, expect, 8, cudaMemcpyDeviceToHost);
        const int heavy = spj_dist_heavy_keys(dj, nullptr, 0);
        const bool ok = n == n_s && got == want;
        printf("check: %s pairs=%lld expected=%lld heavy_keys=%d\n", ok ? "ok" : "MISMATCH", (long long)n,
               (long long)n_s, heavy);
        bad += !ok;
    }
    spj_dist_destroy(dj);
    cudaFree(r);
    cudaFree(s);
    cudaFree(expect);
    cudaFree(sum);
    cudaFree(n_dev);
    return bad ? 1 : 0;
}
