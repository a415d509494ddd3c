// spj_common.h -- types, hashes and the synthetic-data generator shared by the
// host (g++) and device (nvcc) halves of libspidjoin.
//
// The tuple is the reference's kv_pair_t / tuplePair_t (include/type_defs.hpp:53-56,
// src/dpu/include/argument.h:42-46 of yonsei-hpcp/spid-join): {u32 key, u32 payload}.
// Key 0 marks an empty slot or padding and never joins, as in the reference's
// kernels (src/dpu/src/join/glb_partition_packet.c:423, a2a_srj_build.c:246).
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SPJ_HD __host__ __device__ __forceinline__
#else
#define SPJ_HD inline
#endif

namespace spj {

struct alignas(8) Tuple {
    uint32_t key;
    uint32_t pay;
};

// glb_partition_hash of src/dpu/src/hash.c:117-166 (SuperFastHash-style over the
// four key bytes, seed 4, final avalanche). The GPU partitions on its low bits and
// places tuples in the shared-memory table with the bits above them, so the
// partition histogram is bit-identical to the reference's count kernel
// (glb_partition_count.c:190-209) for the same partition count.
SPJ_HD uint32_t glb_partition_hash(uint32_t key) {
    uint32_t h = 4u;
    h += key & 0xffffu;
    uint32_t tmp = (((key >> 16) & 0xffffu) << 11) ^ h;
    h = (h << 16) ^ tmp;
    h += h >> 11;
    h ^= h << 3;
    h += h >> 5;
    h ^= h << 4;
    h += h >> 17;
    h ^= h << 25;
    h += h >> 6;
    return h;
}

// join_hash2 of src/dpu/src/hash.c:85-112 (one-at-a-time over the four
// little-endian key bytes): the slot hash of the reference's non-partitioned
// hash join.
SPJ_HD uint32_t join_hash2(uint32_t key) {
    uint32_t h = 0;
    for (int b = 0; b < 4; b++) {
        h += (key >> (8 * b)) & 0xffu;
        h += h << 10;
        h ^= h >> 6;
    }
    h += h << 3;
    h ^= h >> 11;
    h += h << 15;
    return h;
}

// A selection on a tuple (spj_predicate_t): the comparisons of the reference's
// TPC-H predicates (src/dpu/include/select.h:30-37, PREDINT64) and its inclusive
// range (predi_btw, :44-47) on the key (field 1) or payload (field 2) as
// unsigned 32-bit values; field 0 passes every tuple.
struct Pred {
    uint32_t field, op, lo, hi;
};

SPJ_HD bool pred_pass(const Pred &p, uint32_t key, uint32_t pay) {
    if (p.field == 0) return true;
    const uint32_t v = p.field == 1 ? key : pay;
    switch (p.op) {
        case 0: return v == p.lo;
        case 1: return v <= p.lo;
        case 2: return v >= p.lo;
        case 3: return v < p.lo;
        case 4: return v > p.lo;
        default: return p.lo <= v && v <= p.hi;
    }
}

// splitmix64 (Steele, Lea, Flood 2014): the counter-based mixer of the generator
// and the finaliser of the order-independent output checksum.
SPJ_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

SPJ_HD uint64_t pair_digest(uint32_t lvalue, uint32_t rvalue) {
    return mix64((uint64_t(lvalue) << 32) | rvalue);
}

SPJ_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// ---------------------------------------------------------------- generator --
// Seeded, counter-based generator of the benchmark relations. Every value depends
// only on (seed, index), so the host and the device produce the same R bytes and
// the same uniform S bytes; Zipf S uses double-precision exp/log and is generated
// on one side only (the bytes then travel).

// Pseudo-random permutation of [0, n): a 4-round unbalanced Feistel network on
// ceil(log2 n) bits with cycle-walking back into [0, n).
struct Perm {
    uint64_t n;
    uint64_t seed;
    int lo_bits, hi_bits;
};

SPJ_HD Perm make_perm(uint64_t n, uint64_t seed) {
    Perm p;
    p.n = n;
    p.seed = seed;
    int b = 2;
    while ((1ull << b) < n) b++;
    p.lo_bits = b / 2;
    p.hi_bits = b - p.lo_bits;
    return p;
}

SPJ_HD uint64_t feistel(const Perm &p, uint64_t x) {
    const uint64_t lo_mask = (1ull << p.lo_bits) - 1, hi_mask = (1ull << p.hi_bits) - 1;
    uint64_t lo = x & lo_mask, hi = x >> p.lo_bits;
    for (int r = 0; r < 4; r += 2) {
        hi ^= mix64(p.seed + 0x9e3779b97f4a7c15ull * (uint64_t)(r + 1) + lo) & hi_mask;
        lo ^= mix64(p.seed + 0x9e3779b97f4a7c15ull * (uint64_t)(r + 2) + hi) & lo_mask;
    }
    return (hi << p.lo_bits) | lo;
}

SPJ_HD uint64_t perm_apply(const Perm &p, uint64_t x) {
    uint64_t y = feistel(p, x);
    while (y >= p.n) y = feistel(p, y);
    return y;
}

// Uniform double in [0, 1) from the stream (seed, index, attempt).
SPJ_HD double unit_double(uint64_t seed, uint64_t idx, uint32_t attempt) {
    uint64_t z = mix64(seed ^ mix64(idx * 0x9e3779b97f4a7c15ull + attempt));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Zipf(s) over ranks 1..n by rejection-inversion (W. Hoermann and G. Derflinger,
// "Rejection-inversion to generate variates from monotone discrete distributions",
// ACM TOMACS 6(3), 1996). H is an antiderivative of x^-s; x^(1-s) is evaluated
// through expm1/log1p so s = 1 needs no special case.
struct Zipf {
    double s, h_lo, h_hi, squeeze;
    uint64_t n;
};

SPJ_HD double zipf_ratio_log1p(double x) {  // log1p(x)/x, continuous at 0
    return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
}
SPJ_HD double zipf_ratio_expm1(double x) {  // expm1(x)/x, continuous at 0
    return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + 0.5 * x * (1.0 + (x / 3.0) * (1.0 + 0.25 * x));
}
SPJ_HD double zipf_H(const Zipf &z, double x) {
    double lx = log(x);
    return zipf_ratio_expm1((1.0 - z.s) * lx) * lx;
}
SPJ_HD double zipf_Hinv(const Zipf &z, double y) {
    double t = y * (1.0 - z.s);
    if (t < -1.0) t = -1.0;
    return exp(zipf_ratio_log1p(t) * y);
}
SPJ_HD double zipf_h(const Zipf &z, double x) { return exp(-z.s * log(x)); }

SPJ_HD Zipf make_zipf(uint64_t n, double s) {
    Zipf z;
    z.s = s;
    z.n = n;
    z.h_lo = zipf_H(z, 1.5) - 1.0;
    z.h_hi = zipf_H(z, (double)n + 0.5);
    z.squeeze = 2.0 - zipf_Hinv(z, zipf_H(z, 2.5) - zipf_h(z, 2.0));
    return z;
}

SPJ_HD uint64_t zipf_rank(const Zipf &z, uint64_t seed, uint64_t idx) {
    for (uint32_t a = 0;; a++) {
        double y = z.h_hi + unit_double(seed, idx, a) * (z.h_lo - z.h_hi);
        double x = zipf_Hinv(z, y);
        double kd = x + 0.5;
        uint64_t k = kd < 1.0 ? 1 : (uint64_t)kd;
        if (k > z.n) k = z.n;
        if ((double)k - x <= z.squeeze || y >= zipf_H(z, (double)k + 0.5) - zipf_h(z, (double)k))
            return k;
        if (a > 1000) return k;  // unreachable in practice: acceptance rate > 0.8
    }
}

// The benchmark relations (seeded; payload = row id):
//   R[i] = (1 + perm_R(i), i)                     keys: a permutation of 1..nR
//   S[j] = (R[m(j)].key, j) with m(j) = floor(u * nR) (zipf 0) or
//          perm_rank(zipf_rank(j) - 1) (zipf s > 0; rank order is a second
//          seeded permutation of R, so hot keys spread over all partitions).
// Because R's payload is its row id, the expected join pair of S[j] is (m(j), j).
struct GenSpec {
    uint64_t seed;
    uint64_t nR, nS;
    double zipf_s;
};

SPJ_HD uint64_t seed_R(uint64_t seed) { return mix64(seed ^ 0x52454c4154494f4eull); }
SPJ_HD uint64_t seed_rank(uint64_t seed) { return mix64(seed ^ 0x52414e4b4f524452ull); }
SPJ_HD uint64_t seed_S(uint64_t seed) { return mix64(seed ^ 0x535354524541414dull); }

SPJ_HD Tuple gen_r(const Perm &pr, uint64_t i) {
    Tuple t;
    t.key = (uint32_t)(1 + perm_apply(pr, i));
    t.pay = (uint32_t)i;
    return t;
}

// Row of R matched by S[j].
SPJ_HD uint64_t gen_s_row(const GenSpec &g, const Zipf &z, const Perm &prank, uint64_t j) {
    if (g.zipf_s <= 0.0) return mulhi64(mix64(seed_S(g.seed) ^ (j * 0x9e3779b97f4a7c15ull)), g.nR);
    uint64_t rank = zipf_rank(z, seed_S(g.seed), j);
    return perm_apply(prank, rank - 1);
}

}  // namespace spj
