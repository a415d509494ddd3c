// spj_kernels.cu -- sm_100a kernels of the B200 SPID-Join equi-join.
//
// A plan runs a batch of J joins (J = 1 for the plain join) as one fixed
// sequence of launches, each covering every join, with no host synchronisation:
//
//   k_hist       per-chunk partition histograms of every R and S (one read pass)
//   k_colscan    per-partition exclusive offsets across chunks
//   k_basescan   partition starts (exclusive scan of the totals)
//   k_scatter1   radix scatter pass 1 (coarse buckets; the only pass for <= 256 partitions)
//   k_items      skew-bounded work list of pass 2
//   k_scatter2   radix scatter pass 2 (fine partitions), persistent CTAs
//   k_units      work units: (join, partition, S range); heavy partitions split
//   k_join_*     persistent CTAs over the unit queue: build the R partition's
//                shared-memory structure, probe the unit's S range, emit pairs with
//                warp-aggregated reservations of output chunks (32-1024 pairs)
//   k_fixup_*    per join: move the pairs of partly used last chunks into the
//                holes those chunks left, so the output is dense
//
// This is the B200 form of the reference's pipeline (yonsei-hpcp/spid-join):
// glb_partition_count.c (count), glb_partition_packet.c + the host-mediated
// rotate-and-stream shuffle (scatter; on one GPU the shuffle is the scatter
// itself), a2a_packetwise_srj_local_partition.c + a2a_srj_build.c +
// a2a_srj_probe_inner_mt.c (the local join: a partition here is sized so its
// table fits one CTA's shared memory, so no second local partitioning pass is
// needed), finish_join.c (output framing: dense, no padding).
#include <cuda_runtime.h>

#include "spj_async.cuh"
#include "spj_internal.h"

namespace spj {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Largest r < n with prefix[r] <= x (prefix has n + 1 non-decreasing entries).
__device__ __forceinline__ uint32_t find_slot(const uint32_t *prefix, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Writes the descriptors of a one-join plan from kernel parameters (no host copy)
// and zeroes the execution's counters (the batch counters and the join's, which
// lie next to each other: ctr_words 32-bit words), so an execution needs no
// separate memset. With keep_r, R owns no chunk, partition or coarse bucket of
// the count and scatter grids (its partitions are reused), and every CTA of them
// maps to S.
__global__ void k_init_single(PlanDev P, RelDev r0, RelDev r1, JoinDev j0, uint32_t nch0, uint32_t nch1, uint32_t f,
                              uint32_t f1, bool keep_r, uint32_t ctr_words) {
    uint32_t *ctr = reinterpret_cast<uint32_t *>(P.bctr);
    for (uint32_t i = threadIdx.x; i < ctr_words; i += blockDim.x) ctr[i] = 0u;
    if (threadIdx.x != 0) return;
    P.rel[0] = r0;
    P.rel[1] = r1;
    P.join[0] = j0;
    const uint32_t rch = keep_r ? 0u : nch0, rf = keep_r ? 0u : f, rf1 = keep_r ? 0u : f1;
    P.chunk_prefix[0] = 0;
    P.chunk_prefix[1] = rch;
    P.chunk_prefix[2] = rch + nch1;
    P.part_prefix[0] = 0;
    P.part_prefix[1] = rf;
    P.part_prefix[2] = rf + f;
    P.coarse_prefix[0] = 0;
    P.coarse_prefix[1] = rf1;
    P.coarse_prefix[2] = rf1 + f1;
    P.jpart_prefix[0] = 0;
    P.jpart_prefix[1] = f;
}

// ------------------------------------------------------------ heavy keys --
// SPID-Join spreads a skewed S partition over replicated R tables (rank-set and
// bank-set replication, glb_partition_count.c:317-318,
// glb_chipwise_partition_count.c:251-255). On the GPU the adaptive work units do
// that for every heavy partition; on top of it, the keys that a sample of S
// shows to be frequent are joined on the fly: the count pass over R records one
// R payload per heavy key, and the first scatter pass over S emits the pairs of
// heavy-key S tuples straight into the output instead of partitioning them, so
// those tuples skip the second pass and the join's read.

// A CTA's copy of the heavy table in shared memory, with a 2^14-bit filter of
// the keys' Fibonacci hashes, so that most tuples are told apart from the heavy
// keys by one shared-memory word (a random gather from the global table would
// cost a wavefront per line and compete with the tile sort for the L1 pipe).
struct HeavySmem {
    uint32_t bm[512];        // filter bit (key * 0x9E3779B1) >> 18
    uint32_t key[kHeavySlots];
    uint32_t pay[kHeavySlots];
    uint32_t found[kHeavySlots / 32];
};

// Loads the heavy table of one join into shared memory (all threads; callers
// synchronise before use).
__device__ __forceinline__ void heavy_smem_load(HeavySmem &H, const HeavyTab *hv) {
    for (int i = threadIdx.x; i < 512; i += blockDim.x) H.bm[i] = 0;
    for (int i = threadIdx.x; i < kHeavySlots / 32; i += blockDim.x) H.found[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < kHeavySlots; i += blockDim.x) {
        const uint32_t k = hv->key[i];
        H.key[i] = k;
        H.pay[i] = hv->pay[i];
        if (k) {
            const uint32_t bi = (k * 0x9E3779B1u) >> 18;
            atomicOr(&H.bm[bi >> 5], 1u << (bi & 31));
            if (hv->found[i]) atomicOr(&H.found[i >> 5], 1u << (i & 31));
        }
    }
}

// Slot of a heavy key in the shared-memory table, or -1.
__device__ __forceinline__ int heavy_find(const HeavySmem &H, uint32_t key) {
    const uint32_t prod = key * 0x9E3779B1u;
    const uint32_t bi = prod >> 18;
    if (!((H.bm[bi >> 5] >> (bi & 31)) & 1u)) return -1;
    uint32_t s = prod >> (32 - 9);  // kHeavySlots = 2^9
    for (int i = 0; i < kHeavySlots; i++) {
        const uint32_t k = H.key[s];
        if (k == key) return (int)s;
        if (k == 0) return -1;
        s = (s + 1) & (kHeavySlots - 1);
    }
    return -1;
}

// One CTA per join: samples heavy_sample S keys (one at a pseudo-random position
// inside each of heavy_sample strides of floor(|S| / heavy_sample) tuples),
// counts them in a shared-memory
// table and keeps the keys seen at least T times, T = max(4, sample/16384)
// doubled until at most kHeavyMax keys remain. Which keys are chosen changes only
// the speed, never the result.
__global__ void __launch_bounds__(1024) k_heavy_sample(PlanDev P) {
    extern __shared__ uint32_t smp[];
    uint32_t *sk = smp, *sc = smp + kSampleSlots;
    __shared__ unsigned s_cand, s_n;
    const JoinDev &J = P.join[blockIdx.x];
    HeavyTab *hv = J.heavy;
    if (!hv) return;
    for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) sk[i] = sc[i] = 0;
    for (int i = threadIdx.x; i < kHeavySlots; i += blockDim.x) {
        hv->key[i] = 0;
        hv->found[i] = 0;
    }
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const RelDev &Rs = P.rel[2 * blockIdx.x + 1];
    const uint64_t n = Rs.n;
    const uint32_t m = (uint32_t)min((uint64_t)J.heavy_sample, n);
    const uint64_t stride = m ? n / m : 1;  // one division; the sample's positions need none
    constexpr int U = 8;  // loads in flight per thread
    for (uint32_t i0 = threadIdx.x; i0 < m; i0 += U * blockDim.x) {
        uint32_t key[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const uint32_t i = i0 + k * blockDim.x;
            key[k] = 0;
            if (i < m) {
                const uint64_t idx = (uint64_t)i * stride + mulhi64(mix64(i * 0x9e3779b97f4a7c15ull + n), stride);
                const Tuple t = Rs.in[idx];
                key[k] = pred_pass(Rs.pred, t.key, t.pay) ? t.key : 0u;
            }
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            // lanes holding the same key add to its counter once (a hot key's
            // counter would otherwise take thousands of serialised atomics)
            const unsigned same = __match_any_sync(0xffffffffu, key[k]);
            if (!key[k] || (threadIdx.x & 31) != (unsigned)(__ffs(same) - 1)) continue;
            uint32_t sl = (key[k] * 0x9E3779B1u) >> (32 - 14);  // kSampleSlots = 2^14
            for (int step = 0; step < 16; step++) {  // a full neighbourhood drops the sample
                const uint32_t prev = atomicCAS(&sk[sl], 0u, key[k]);
                if (prev == 0u || prev == key[k]) {
                    atomicAdd(&sc[sl], (uint32_t)__popc(same));
                    break;
                }
                sl = (sl + 1) & (kSampleSlots - 1);
            }
        }
    }
    uint32_t T = max(4u, m >> 14);
    for (int iter = 0; iter < 24; iter++) {
        __syncthreads();
        if (threadIdx.x == 0) s_cand = 0;
        __syncthreads();
        unsigned c = 0;
        for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) c += sc[i] >= T ? 1u : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cand, c);
        __syncthreads();
        if (s_cand <= (unsigned)kHeavyMax) break;
        T *= 2;
    }
    // automatic mode: the heavy-key path pays only when the heavy keys hold most of
    // S (every tuple then takes a filter lookup in the count and first scatter
    // passes); below kHeavyMinShare of the sample it stays off
    if (threadIdx.x == 0) s_cand = 0;
    __syncthreads();
    {
        unsigned c = 0;
        for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) c += sc[i] >= T ? sc[i] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cand, c);
    }
    __syncthreads();
    if (J.heavy_auto && (double)s_cand < kHeavyMinShare * (double)m) T = 0xffffffffu;
    for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) {
        const uint32_t key = sk[i];
        if (!key || sc[i] < T || atomicAdd(&s_n, 1u) >= (unsigned)kHeavyMax) continue;
        uint32_t sl = (key * 0x9E3779B1u) >> (32 - 9);
        for (int step = 0; step < kHeavySlots && atomicCAS(&hv->key[sl], 0u, key) != 0u; step++)
            sl = (sl + 1) & (kHeavySlots - 1);  // at most 256 of the 512 slots are taken
    }
    __syncthreads();
    if (threadIdx.x == 0) hv->n = min(s_n, (unsigned)kHeavyMax);
}

// ------------------------------------------------------------- histogram --
// glb_partition_count.c:119-236 on B200: each CTA counts one contiguous chunk
// into a shared-memory histogram; key-0 tuples are skipped (:190-192).
__global__ void __launch_bounds__(kHistThreads) k_hist(PlanDev P) {
    extern __shared__ uint32_t sh[];
    const uint32_t r = find_slot(P.chunk_prefix, P.nrel, blockIdx.x);
    const uint32_t c = blockIdx.x - P.chunk_prefix[r];
    const RelDev R = P.rel[r];
    const int bits = P.join[R.join].bits, b2 = P.join[R.join].fine_bits;
    const uint32_t F = 1u << bits, mask = F - 1;
    for (uint32_t i = threadIdx.x; i < F; i += blockDim.x) sh[i] = 0;
    // heavy keys: R records one payload per heavy key, S leaves them out of its
    // partitions (the first scatter pass joins them on the fly)
    HeavyTab *hv = P.join[R.join].heavy;
    const int hmode = (hv && hv->n) ? ((r & 1u) ? 2 : 1) : 0;  // 1: R, 2: S
    HeavySmem &HS = *reinterpret_cast<HeavySmem *>(sh + F);
    if (hmode) heavy_smem_load(HS, hv);
    __syncthreads();
    const uint32_t b = c * R.chunk;
    const uint32_t e = min(R.n, b + R.chunk);
    auto count = [&](uint32_t key, uint32_t pay) {
        if (!key || !pred_pass(R.pred, key, pay)) return;
        if (hmode) {
            const int hs = heavy_find(HS, key);
            if (hs >= 0) {
                if (hmode == 2) return;
                if (atomicCAS(&hv->found[hs], 0u, 1u) == 0u) hv->pay[hs] = pay;
            }
        }
        atomicAdd(&sh[glb_partition_hash(key) & mask], 1u);
    };
    if (b < e) {
        const uint4 *in2 = reinterpret_cast<const uint4 *>(R.in);
        const uint32_t b2i = b >> 1, e2 = e >> 1;
        constexpr int U = 4;
        // software-pipelined: the next group's loads are in flight while this
        // group is counted
        uint4 v[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const uint32_t j = b2i + threadIdx.x + k * blockDim.x;
            v[k] = j < e2 ? __ldcs(in2 + j) : make_uint4(0, 0, 0, 0);
        }
        for (uint32_t i = b2i + threadIdx.x; i < e2; i += U * blockDim.x) {
            uint4 nx[U];
#pragma unroll
            for (int k = 0; k < U; k++) {
                const uint32_t j = i + (U + k) * blockDim.x;
                nx[k] = j < e2 ? __ldcs(in2 + j) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int k = 0; k < U; k++) {
                count(v[k].x, v[k].y);
                count(v[k].z, v[k].w);
            }
#pragma unroll
            for (int k = 0; k < U; k++) v[k] = nx[k];
        }
        if ((e & 1u) && threadIdx.x == 0) {
            const Tuple t = R.in[e - 1];
            count(t.key, t.pay);
        }
    }
    __syncthreads();
    uint32_t *out = R.hist + (size_t)c * F;
    for (uint32_t i = threadIdx.x; i < F; i += blockDim.x) out[i] = sh[i];
    if (b2 > 0) {  // per-chunk counts of the coarse buckets (the pass-2 work list)
        const uint32_t f1 = F >> b2, q_per = 1u << b2;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (uint32_t cb = warp; cb < f1; cb += blockDim.x >> 5) {
            uint32_t sum = 0;
            for (uint32_t q = lane; q < q_per; q += 32) sum += sh[(cb << b2) + q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) R.chist[(size_t)c * f1 + cb] = sum;
        }
    }
}

// Per partition: exclusive offsets of each chunk inside the partition (in place)
// and the partition total.
__global__ void k_colscan(PlanDev P) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.total_parts) return;
    const uint32_t r = find_slot(P.part_prefix, P.nrel, t);
    const RelDev R = P.rel[r];
    const uint32_t F = 1u << P.join[R.join].bits;
    const uint32_t p = t - P.part_prefix[r];
    uint32_t run = 0, c = 0;
    uint32_t *col = R.hist + p;
    for (; c + 8 <= R.nchunks; c += 8) {  // eight loads in flight before the stores
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = col[(size_t)(c + k) * F];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            col[(size_t)(c + k) * F] = run;
            run += v[k];
        }
    }
    for (; c < R.nchunks; c++) {
        const uint32_t v = col[(size_t)c * F];
        col[(size_t)c * F] = run;
        run += v;
    }
    R.total[p] = run;
}

// Block-wide exclusive scan of up to 1024 * 32 totals (one CTA per relation).
__global__ void __launch_bounds__(1024) k_basescan(PlanDev P) {
    __shared__ uint32_t warp_sums[32];
    const RelDev R = P.rel[blockIdx.x];
    const uint32_t F = 1u << P.join[R.join].bits;
    const uint32_t per = (F + blockDim.x - 1) / blockDim.x;
    const uint32_t beg = threadIdx.x * per, end = min(F, beg + per);
    uint32_t sum = 0, mx = 0;
    for (uint32_t i = beg; i < end; i++) {
        const uint32_t v = R.total[i];
        sum += v;
        mx = max(mx, v);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_sums[lane] = wi - w;
    }
    __syncthreads();
    uint32_t run = warp_sums[warp] + incl - sum;
    for (uint32_t i = beg; i < end; i++) {
        const uint32_t v = R.total[i];
        R.base[i] = run;
        run += v;
    }
    JoinCtr *jc = P.join[R.join].ctr;
    if (lane == 0) atomicMax((blockIdx.x & 1) == 0 ? &jc->max_r_part : &jc->max_s_part, mx);
}

// --------------------------------------------------------------- scatter --
// The partition id p = glb_partition_hash(key) & (F-1) is split into a coarse
// bucket (its high b1 bits) and a fine bucket (its low b2 bits). Pass 1 moves
// every chunk's tuples to their coarse region, pass 2 every (chunk, coarse)
// segment to its final fine positions; with b2 = 0 pass 1 is the only pass. No
// pass has more than 256 buckets, and each CTA sorts a 4096-tuple tile by bucket
// in shared memory before it writes, so stores leave in runs of ~16-32 tuples
// (128-256 bytes) and only #CTAs x 256 write fronts are open at any time --
// few enough to stay in L2. Positions are exact (from the count pass): no global
// atomics. This replaces glb_partition_packet.c:420-464 and the host-mediated
// rotate-and-stream shuffle (queryHostFunc.cc:481-777); on one GPU the shuffle
// is the scatter itself.
struct __align__(128) TileSmem {
    Tuple inbuf[2][kTile];     // bulk-copy double buffer of input tiles
    Tuple stage[kTile + 256];  // tile sorted by bucket (+1 spare slot per bucket with bulk stores)
    union {                    // one write-out per call, so the two sets share memory
        struct {
            uint8_t bkt[kTile];    // element stores: bucket of each stage slot
            uint32_t wpos[256];    // element stores: global position of stage slot j is wpos[b] + j
        };
        struct {
            uint32_t len[256];     // bulk stores: the bucket's tuples in this tile
            uint32_t gpos[256];    // bulk stores: global position of the bucket's first tuple
        };
    };
    uint32_t cnt[256];
    uint32_t off[256];         // stage slot of the bucket's first tuple in this tile
    uint32_t cursor[256];
    uint64_t bar[2];
    uint32_t valid;
    uint32_t seg_begin, seg_len;
    uint32_t item;
    uint32_t hcnt;             // heavy pairs of the tile being ranked
    uint32_t hoff, hlen, hpos; // the tile's heavy pairs: stage slot, count, output position
};

// Two scatter CTAs fit one SM's 228 KiB of shared memory (1 KiB of it reserved
// per CTA), with the heavy table's copy as well.
static_assert(2 * (sizeof(TileSmem) + sizeof(HeavySmem) + 1024) <= 228 * 1024, "two scatter CTAs per SM");

// Where heavy-key S tuples go in the first scatter pass over S: their pairs are
// appended to the join's output (positions reserved per tile with one atomic).
struct HeavyOut {
    const HeavySmem *hs;
    uint2 *out;
    uint32_t cap;
    JoinCtr *ctr;
    int keep_unmatched;  // SMJ/NL keep an unmatched S tuple as it is
};

// The output value of heavy-key S tuple t (slot hs): its pair, the tuple itself
// when unmatched and kept, or nothing (false).
__device__ __forceinline__ bool heavy_value(const HeavyOut &h, int hs, Tuple &t) {
    if ((h.hs->found[hs >> 5] >> (hs & 31)) & 1u) {
        t.key = h.hs->pay[hs];
        return true;
    }
    return h.keep_unmatched != 0;
}

// Scatters in[b, e) to out[cursor[bucket] ...], advancing the cursors. Input
// tiles arrive by bulk copy (TMA) into a double buffer, so the next tile is in
// flight while this one is sorted and written. A tuple at an odd boundary index
// is moved with an ordinary load (bulk copies need 16-byte alignment).
// Each tile is counting-sorted by bucket in shared memory, then written out in
// one of two ways (kBulk):
//  * element stores: one stage slot per thread, consecutive threads write a
//    bucket's run with coalesced stores;
//  * bulk stores: each bucket's run starts at a stage slot of the same 16-byte
//    parity as its global address (the spare slot per bucket absorbs the shift)
//    and leaves as one bulk store (TMA) of its aligned body, plus at most one
//    ordinary store at each end, issued by the bucket's thread. The writer
//    threads' proxy fence is the price; long runs (hot buckets) repay it.
// Returns false (the same value in every thread) when a bulk copy timed out.
// With kHeavy (the first pass over S of a join with heavy keys) a tuple whose key
// is in the heavy table does not go to a bucket: its output value is staged
// after the buckets' runs and written to the join's output (see HeavyOut).
// The tile's heavy pairs, staged at [hoff, hoff + hlen), to the join's output at
// hpos (coalesced stores by all threads; called after the stage barrier).
__device__ __forceinline__ void write_heavy_run(const TileSmem &S, const HeavyOut &h) {
    const uint32_t n = S.hlen, off = S.hoff, pos = S.hpos;
    const uint2 *st2 = reinterpret_cast<const uint2 *>(S.stage);
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        if (pos + j < h.cap)
            h.out[pos + j] = st2[off + j];
        else
            atomicOr(&h.ctr->error, 2u);
    }
}

template <bool kHot, bool kBulk, bool kHeavy = false, typename BucketFn>
__device__ __forceinline__ bool scatter_range(const Tuple *__restrict__ in, uint32_t b, uint32_t e,
                                              Tuple *__restrict__ out, TileSmem &S, int nb, BucketFn bucket_of,
                                              uint32_t (&uses)[2], unsigned int *err,
                                              const HeavyOut *hvo = nullptr, const Pred pred = Pred{0u, 0u, 0u, 0u}) {
    constexpr int PER = kTile / kScatterThreads;
    constexpr uint32_t kBulkMin = 8;  // bulk-store bodies shorter than this go by ordinary stores
    uint2 *o2 = reinterpret_cast<uint2 *>(out);
    const uint2 *st2 = reinterpret_cast<const uint2 *>(S.stage);
    const uint32_t par0 = (uint32_t)(reinterpret_cast<uintptr_t>(out) >> 3) & 1u;  // address parity of out[0]
    const bool writer = kBulk && (int)threadIdx.x < nb;
    if (b >= e) return true;
    if (threadIdx.x < 2) {  // boundary tuples at odd indices
        const bool head = threadIdx.x == 0;
        const uint32_t idx = head ? b : e - 1;
        // head: index b when odd; tail: index e-1 when e is odd, unless that is the head
        if ((head && (b & 1u)) || (!head && (e & 1u) && !((b & 1u) && e - 1 == b))) {
            Tuple t = in[idx];
            if (!pred_pass(pred, t.key, t.pay)) t.key = 0;  // not selected
            int hs = -1;
            if (kHeavy && t.key) hs = heavy_find(*hvo->hs, t.key);
            if (hs >= 0) {
                if (heavy_value(*hvo, hs, t)) {
                    const uint32_t pos = (uint32_t)atomicAdd(&hvo->ctr->out_reserved, 1ull);
                    if (pos < hvo->cap)
                        hvo->out[pos] = make_uint2(t.key, t.pay);
                    else
                        atomicOr(&hvo->ctr->error, 2u);
                    atomicAdd(&hvo->ctr->heavy_tuples, 1ull);
                }
            } else if (t.key) {
                const uint32_t pos = atomicAdd(&S.cursor[bucket_of(t.key)], 1u);
                o2[pos] = make_uint2(t.key, t.pay);
            }
        }
    }
    __syncthreads();
    const uint32_t tb = b + (b & 1u), te = e - (e & 1u);
    if (tb >= te) return true;
    const uint32_t ntiles = (te - tb + kTile - 1) / kTile;
    if (threadIdx.x == 0) {
        const uint32_t n0 = min((uint32_t)kTile, te - tb);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&S.bar[0], n0 * 8);
        bulk_load(S.inbuf[0], in + tb, n0 * 8, &S.bar[0]);
    }
    for (uint32_t t = 0; t < ntiles; t++) {
        const int buf = t & 1;
        const uint32_t t0 = tb + t * kTile;
        const uint32_t nt = min((uint32_t)kTile, te - t0);
        if (threadIdx.x == 0 && t + 1 < ntiles) {
            const uint32_t t1 = t0 + kTile, n1 = min((uint32_t)kTile, te - t1);
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&S.bar[buf ^ 1], n1 * 8);
            bulk_load(S.inbuf[buf ^ 1], in + t1, n1 * 8, &S.bar[buf ^ 1]);
        }
        const bool ok = mbar_wait(&S.bar[buf], uses[buf] & 1u, err);
        uses[buf]++;
        if (__syncthreads_or(!ok)) {  // a copy timed out (error bit set): all threads stop alike
            // copies already issued may still land: give them a bounded wait before leaving
            if (threadIdx.x == 0 && t + 1 < ntiles) mbar_wait(&S.bar[buf ^ 1], uses[buf ^ 1] & 1u, err);
            if (writer) bulk_wait_all();
            return false;
        }
        Tuple v[PER];
        uint32_t br[PER];  // bucket << 16 | rank inside the tile; 0xffff0000 = no tuple
        // Rank. In a hot run (kHot: a pass-2 segment of one heavy chunk, where a
        // hot key puts most tuples in one bucket) a warp whose 32 tuples share a
        // bucket takes its 32 ranks with one counter increment instead of 32
        // serialised ones; elsewhere the check would only cost time.
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t idx = threadIdx.x + k * kScatterThreads;
            v[k] = idx < nt ? S.inbuf[buf][idx] : Tuple{0u, 0u};
            if (pred.field && !pred_pass(pred, v[k].key, v[k].pay)) v[k].key = 0;  // not selected
            if (kHeavy) {  // heavy key: rank among the tile's heavy pairs (one counter add per warp)
                int hs = v[k].key ? heavy_find(*hvo->hs, v[k].key) : -1;
                const bool isH = hs >= 0;
                const bool emit = isH && heavy_value(*hvo, hs, v[k]);
                const unsigned hm = __ballot_sync(0xffffffffu, emit);
                if (hm) {
                    const int leader = __ffs(hm) - 1;
                    uint32_t base = 0;
                    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&S.hcnt, (uint32_t)__popc(hm));
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (emit) {
                        br[k] = 0xfffe0000u | (base + __popc(hm & lanemask_lt()));
                        continue;
                    }
                }
                if (isH) {  // heavy and unmatched, not kept: dropped
                    br[k] = 0xffff0000u;
                    continue;
                }
            }
            const uint32_t bk = v[k].key ? (uint32_t)bucket_of(v[k].key) : 0xffffu;
            if (kHot) {
                const uint32_t b0 = __shfl_sync(0xffffffffu, bk, 0);
                if (__all_sync(0xffffffffu, bk == b0) && b0 != 0xffffu) {
                    uint32_t base = 0;
                    if ((threadIdx.x & 31) == 0) base = atomicAdd(&S.cnt[b0], 32u);
                    br[k] = (b0 << 16) | (__shfl_sync(0xffffffffu, base, 0) + (threadIdx.x & 31));
                    continue;
                }
            }
            br[k] = bk != 0xffffu ? (bk << 16) | atomicAdd(&S.cnt[bk], 1u) : 0xffff0000u;
        }
        if (writer) bulk_wait_read();  // the previous tile's bulk stores have read the stage
        __syncthreads();
        if (threadIdx.x < 32) {  // exclusive scan of the <= 256 bucket counts (+1 each with bulk stores)
            const int lane = threadIdx.x;
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int j = lane * 8 + i;
                c[i] = j < nb ? S.cnt[j] : 0;
                sum += j < nb ? c[i] + (kBulk ? 1u : 0u) : 0u;
            }
            uint32_t incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
            }
            uint32_t run = incl - sum;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int j = lane * 8 + i;
                if (j < nb) {
                    const uint32_t g = S.cursor[j];
                    if (kBulk) {
                        S.off[j] = run + ((run ^ (g + par0)) & 1u);
                        S.len[j] = c[i];
                        S.gpos[j] = g;
                        run += c[i] + 1;
                    } else {
                        S.off[j] = run;
                        S.wpos[j] = g - run;
                        run += c[i];
                    }
                    S.cursor[j] = g + c[i];
                    S.cnt[j] = 0;
                }
            }
            if (!kBulk && lane == 31) S.valid = incl;
            if (kHeavy && lane == 31) {  // heavy pairs after the buckets' runs
                const uint32_t h = S.hcnt;
                S.hoff = incl;
                S.hlen = h;
                S.hcnt = 0;
                if (h) {
                    S.hpos = (uint32_t)atomicAdd(&hvo->ctr->out_reserved, (unsigned long long)h);
                    atomicAdd(&hvo->ctr->heavy_tuples, (unsigned long long)h);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t bk = br[k] >> 16;
            if (kHeavy && bk == 0xfffeu) {
                S.stage[S.hoff + (br[k] & 0xffffu)] = v[k];
            } else if (bk != 0xffffu) {
                const uint32_t slot = S.off[bk] + (br[k] & 0xffffu);
                S.stage[slot] = v[k];
                if (!kBulk) S.bkt[slot] = (uint8_t)bk;
            }
        }
        if (kBulk) {
            fence_proxy_async_smem();  // the stage writes before the bulk stores that read them
            __syncthreads();
            if (writer) {  // bucket threadIdx.x's run of this tile
                uint32_t c = S.len[threadIdx.x];
                if (c) {
                    uint32_t g = S.gpos[threadIdx.x], sl = S.off[threadIdx.x];
                    if ((g + par0) & 1u) {  // head tuple up to the 16-byte boundary
                        o2[g++] = st2[sl++];
                        c--;
                    }
                    const uint32_t body = c & ~1u;
                    if (body >= kBulkMin) {
                        bulk_store(o2 + g, st2 + sl, body * 8);
                        bulk_commit();
                    } else {
                        for (uint32_t i = 0; i < body; i++) o2[g + i] = st2[sl + i];
                    }
                    if (c & 1u) o2[g + body] = st2[sl + body];
                }
            }
            // the next tile's rank phase may start: counts are zero, and the stage
            // is rewritten only after its writers' bulk stores have read it
            if (kHeavy) write_heavy_run(S, *hvo);
        } else {
            __syncthreads();
            // write phase, unrolled so all shared loads are in flight before the stores
            const uint32_t valid = S.valid;
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t j = threadIdx.x + k * kScatterThreads;
                if (j < valid) {
                    v[k] = S.stage[j];
                    br[k] = S.bkt[j];
                }
            }
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t j = threadIdx.x + k * kScatterThreads;
                if (j < valid) br[k] = S.wpos[br[k]] + j;
            }
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t j = threadIdx.x + k * kScatterThreads;
                if (j < valid) o2[br[k]] = make_uint2(v[k].key, v[k].pay);
            }
            if (kHeavy) write_heavy_run(S, *hvo);
            // the next tile's rank phase may start: counts are zero, and its first
            // barrier orders these reads of stage/wpos before they are rewritten
        }
    }
    if (writer) bulk_wait_read();
    return true;
}

// Bulk stores pay for their proxy fence once runs average 32 tuples or more:
// passes of at most 128 buckets, and pass-2 segments of one heavy chunk.
constexpr int kBulkMaxBuckets = 128;

__device__ __forceinline__ void tile_init(TileSmem &S) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) S.cnt[i] = 0;
    if (threadIdx.x == 0) S.hcnt = 0;
    if (threadIdx.x == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
}

// Pass 1: one CTA per chunk. Coarse bucket P = p >> b2; the write cursor of
// (chunk c, bucket P) is base[P << b2] + sum_q off[c][(P << b2) + q].
// Pass 1: one CTA per chunk. Coarse bucket P = p >> b2; the write cursor of
// (chunk c, bucket P) is base[P << b2] + sum_q off[c][(P << b2) + q].
// kHeavyJoins = false covers the joins without heavy keys this execution, true
// (launched only for plans that sample heavy keys) the joins with them, whose S
// chunks join their heavy-key tuples on the fly; so the kernel of the common
// case carries none of the heavy-key code, and a join's R and S chunks still
// run in one launch.
template <bool kHeavyJoins>
__global__ void __launch_bounds__(kScatterThreads, kScatterBlocksPerSM) k_scatter1(PlanDev P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    const uint32_t r = find_slot(P.chunk_prefix, P.nrel, blockIdx.x);
    const uint32_t c = blockIdx.x - P.chunk_prefix[r];
    const RelDev R = P.rel[r];
    const JoinDev &J = P.join[R.join];
    if ((J.heavy && J.heavy->n) != kHeavyJoins) return;
    const int bits = J.bits, b2 = J.fine_bits;
    const uint32_t F = 1u << bits, mask = F - 1;
    const int nb = 1 << (bits - b2);
    const int q_per = 1 << b2;
    const uint32_t *off = R.hist + (size_t)c * F;
    tile_init(S);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = warp; b < nb; b += kScatterThreads / 32) {
        uint32_t sum = 0;
        for (int q = lane; q < q_per; q += 32) sum += off[(b << b2) + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) S.cursor[b] = R.base[b << b2] + sum;
    }
    const bool heavy = kHeavyJoins && (r & 1u);  // the S of a join with heavy keys
    HeavySmem &HS = *reinterpret_cast<HeavySmem *>(smem_raw + sizeof(TileSmem));
    if (heavy) heavy_smem_load(HS, J.heavy);
    __syncthreads();
    const uint32_t b0 = c * R.chunk;
    const uint32_t e0 = min(R.n, b0 + R.chunk);
    Tuple *dst = b2 ? R.tmp : R.out;
    uint32_t uses[2] = {0, 0};
    auto coarse = [=](uint32_t key) { return (int)((glb_partition_hash(key) & mask) >> b2); };
    if (heavy) {
        const HeavyOut hvo{&HS, reinterpret_cast<uint2 *>(J.out), (uint32_t)J.out_cap, J.ctr, J.keep_unmatched};
        if (nb <= kBulkMaxBuckets)
            scatter_range<false, true, kHeavyJoins>(R.in, b0, e0, dst, S, nb, coarse, uses, &J.ctr->error, &hvo,
                                                    R.pred);
        else
            scatter_range<false, false, kHeavyJoins>(R.in, b0, e0, dst, S, nb, coarse, uses, &J.ctr->error, &hvo,
                                                     R.pred);
    } else if (nb <= kBulkMaxBuckets) {
        scatter_range<false, true>(R.in, b0, e0, dst, S, nb, coarse, uses, &J.ctr->error, nullptr, R.pred);
    } else {
        scatter_range<false, false>(R.in, b0, e0, dst, S, nb, coarse, uses, &J.ctr->error, nullptr, R.pred);
    }
    bulk_wait_all();  // this thread's bulk stores are performed before the CTA retires
}

// Work list of pass 2: for every (relation, coarse bucket), runs of consecutive
// chunks. A run ends at each chunk where the bucket's running tuple count
// crosses a multiple of `item_target` (and at the last chunk, if tuples remain),
// so runs hold about item_target tuples and a heavy single segment is its own
// run. Within a coarse region the chunks' segments follow each other in chunk
// order, as do the fine offsets, so cursors set from a run's first chunk stay
// exact. One warp per (relation, coarse bucket), 32 chunks per step.
__global__ void k_items(PlanDev P) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= P.total_coarse) return;  // whole warps leave together
    const uint32_t r = find_slot(P.coarse_prefix, P.nrel, t);
    const uint32_t cb = t - P.coarse_prefix[r];
    const RelDev R = P.rel[r];
    const JoinDev &J = P.join[R.join];
    const uint32_t f1 = 1u << (J.bits - J.fine_bits);
    const unsigned long long T = J.item_target;
    const uint32_t nch = R.nchunks;
    unsigned long long carry = 0, cum_last_b = 0;  // count before this step; count at the last run end
    int last_b = -1;                                 // chunk of the last run end
    for (uint32_t base = 0; base < nch; base += 32) {
        const uint32_t c = base + lane;
        const unsigned long long cnt = c < nch ? R.chist[(size_t)c * f1 + cb] : 0u;
        unsigned long long incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const unsigned long long cum = carry + incl, prev = cum - cnt;
        const bool cross = c < nch && cum / T != prev / T;
        // the run ending here starts after the previous run end (this step or earlier)
        const unsigned below = __ballot_sync(0xffffffffu, cross) & ((1u << lane) - 1u);
        const int pl = below ? 31 - __clz(below) : -1;
        const unsigned long long cum_pl = __shfl_sync(0xffffffffu, cum, pl < 0 ? 0 : pl);
        const int start_b = pl >= 0 ? (int)base + pl : last_b;
        const unsigned long long cum_start = pl >= 0 ? cum_pl : cum_last_b;
        const bool tail = c + 1 == nch && !cross && cum > cum_start;
        if (cross || tail) {
            const unsigned i = atomicAdd(&P.bctr->item_count, 1u);
            // a run of one chunk holding a whole item's worth is a hot key's segment
            const bool hot = start_b + 1 == (int)c && cnt >= T;
            if (i < P.max_items)
                P.items[i] = make_uint4(r | (hot ? 0x80000000u : 0u), cb, (uint32_t)(start_b + 1), c + 1);
            else
                atomicOr(&J.ctr->error, 4u);
        }
        const unsigned all = __ballot_sync(0xffffffffu, cross);
        if (all) {
            const int hb = 31 - __clz(all);
            cum_last_b = __shfl_sync(0xffffffffu, cum, hb);
            last_b = (int)base + hb;
        }
        carry = __shfl_sync(0xffffffffu, cum, 31);
    }
}

// Pass 2: persistent CTAs over the work list; each item scatters one run of a
// coarse region to the final fine positions.
__global__ void __launch_bounds__(kScatterThreads, kScatterBlocksPerSM) k_scatter2(PlanDev P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    tile_init(S);
    uint32_t uses[2] = {0, 0};
    const unsigned n_items = min(*(volatile unsigned *)&P.bctr->item_count, P.max_items);
    for (;;) {
        if (threadIdx.x == 0) {
            S.item = atomicAdd(&P.bctr->item_next, 1u);
            S.seg_begin = 0;
            S.seg_len = 0;
        }
        __syncthreads();
        const unsigned it = S.item;
        if (it >= n_items) break;
        const uint4 item = P.items[it];
        const bool hot = (item.x >> 31) != 0;
        const RelDev R = P.rel[item.x & 0x7fffffffu];
        const JoinDev &J = P.join[R.join];
        const int b2 = J.fine_bits;
        const uint32_t F = 1u << J.bits;
        const int nb = 1 << b2;
        const uint32_t qmask = (uint32_t)nb - 1;
        const uint32_t cb = item.y, c0 = item.z, c1 = item.w;
        const uint32_t *off = R.hist + (size_t)c0 * F;
        const uint32_t *nxt = c1 < R.nchunks ? R.hist + (size_t)c1 * F : R.total;
        uint32_t mine_off = 0, mine_cnt = 0;
        for (int q = threadIdx.x; q < nb; q += kScatterThreads) {
            const uint32_t p = (cb << b2) + q;
            const uint32_t o = off[p];
            mine_off += o;
            mine_cnt += nxt[p] - o;
            S.cursor[q] = R.base[p] + o;
        }
        if (mine_off) atomicAdd(&S.seg_begin, mine_off);
        if (mine_cnt) atomicAdd(&S.seg_len, mine_cnt);
        __syncthreads();
        const uint32_t beg = R.base[cb << b2] + S.seg_begin;
        auto fine = [=](uint32_t key) { return (int)(glb_partition_hash(key) & qmask); };
        const uint32_t e2 = beg + S.seg_len;
        const bool ok = hot ? scatter_range<true, true>(R.tmp, beg, e2, R.out, S, nb, fine, uses, &J.ctr->error)
                        : nb <= kBulkMaxBuckets
                            ? scatter_range<false, true>(R.tmp, beg, e2, R.out, S, nb, fine, uses, &J.ctr->error)
                            : scatter_range<false, false>(R.tmp, beg, e2, R.out, S, nb, fine, uses, &J.ctr->error);
        __syncthreads();
        if (!ok) break;
    }
    bulk_wait_all();  // this thread's bulk stores are performed before the CTA retires
}

// ----------------------------------------------------------------- units --
// One warp per (join, partition). The reference replicates every R partition to
// rank_set x bank_set DPUs and splits S among the replicas by element index
// (glb_partition_count.c:317-318, glb_chipwise_partition_count.c:251-255);
// here the replicas are work units, each a CTA that builds the same table and
// probes a contiguous slice of the partition's S.
// Number of units of flat partition t of join j (0 when there is nothing to join).
__device__ __forceinline__ uint32_t unit_count_of(const PlanDev &P, uint32_t j, uint32_t p, uint32_t &ns,
                                                  uint32_t &s0) {
    const JoinDev &J = P.join[j];
    const RelDev &Rr = P.rel[2 * j], &Rs = P.rel[2 * j + 1];
    uint32_t nr;
    if (J.alg == SPJ_ALG_NPHJ) {  // no partitions: units are raw ranges of S
        if (p > 0) return 0;
        nr = Rr.n;
        ns = Rs.n;
        s0 = 0;
    } else {
        nr = Rr.total[p];
        ns = Rs.total[p];
        s0 = Rs.base[p];
    }
    if (ns == 0) return 0;
    if (nr == 0 && !J.keep_unmatched) return 0;
    uint32_t g;
    if (J.skew_mode == SPJ_SKEW_FIXED && J.alg != SPJ_ALG_NPHJ) {
        g = (uint32_t)max(J.group, 1);
    } else {
        g = 1;
        if (ns > J.unit_tuples) {
            g = (ns + J.unit_tuples - 1) / J.unit_tuples;
            g = max(g, (uint32_t)max(J.group, 1));
        }
    }
    return min(g, ns);
}

// Units, step 1: every (join, partition) adds its unit count to its join.
__global__ void k_units_count(PlanDev P) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.total_jparts) return;
    const uint32_t j = find_slot(P.jpart_prefix, P.njoin, t);
    uint32_t ns = 0, s0 = 0;
    const uint32_t g = unit_count_of(P, j, t - P.jpart_prefix[j], ns, s0);
    if (g) atomicAdd(&P.join[j].ctr->units, g);
}

// Units, step 2: each join's units get a contiguous range of the queue, so a
// CTA meets every join in one stretch (at most one output hole per warp and
// join), and each local-join algorithm's joins come in one stretch of their own
// (alg_begin), which that algorithm's kernel works through.
__global__ void __launch_bounds__(1024) k_units_scan(PlanDev P) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t s_carry;
    const uint32_t J = P.njoin;
    const uint32_t per = (J + blockDim.x - 1) / blockDim.x;
    const uint32_t beg = threadIdx.x * per, end = min(J, beg + per);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    for (int A = 0; A < 4; A++) {
        __syncthreads();
        if (threadIdx.x == 0) P.bctr->alg_begin[A] = s_carry;
        if (!(P.alg_mask & (1 << A))) continue;  // uniform: no join uses A
        uint32_t sum = 0;
        for (uint32_t j = beg; j < end; j++)
            if (P.join[j].alg == A) sum += P.join[j].ctr->units;
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        uint32_t total = 0;
        if (warp == 0) {
            const uint32_t w = warp_sums[lane];
            uint32_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += x;
            }
            warp_sums[lane] = wi - w;
            total = __shfl_sync(0xffffffffu, wi, 31);
        }
        __syncthreads();
        uint32_t run = s_carry + warp_sums[warp] + incl - sum;
        for (uint32_t j = beg; j < end; j++) {
            if (P.join[j].alg != A) continue;
            JoinCtr *c = P.join[j].ctr;
            c->unit_base = run;
            run += c->units;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        P.bctr->alg_begin[4] = s_carry;
        P.bctr->unit_count = s_carry;
    }
    for (uint32_t j = beg; j < end; j++) {
        const JoinDev &J = P.join[j];
        JoinCtr *c = J.ctr;
        // the pairs of heavy keys, appended by the first scatter pass, end on a
        // whole output chunk, so every join chunk is aligned; the rest of their
        // last chunk is a hole for the fix-up
        if (J.heavy) {
            c->heavy_keys = J.heavy->n;
            const unsigned long long H = c->out_reserved, ch = J.out_chunk;
            const unsigned long long A = (H + ch - 1) / ch * ch;
            if (A > H) {
                const unsigned h = atomicAdd(&c->hole_count, 1u);
                if (h < kMaxHoles) {
                    J.holes[h].begin = H;
                    J.holes[h].end = A;
                } else {
                    atomicOr(&c->error, 8u);
                }
                c->out_reserved = A;
            }
        }
    }
}

// Units, step 3: one warp per (join, partition) writes its units. The reference
// replicates every R partition to rank_set x bank_set DPUs and splits S among
// the replicas by element index (glb_partition_count.c:317-318,
// glb_chipwise_partition_count.c:251-255); here the replicas are work units,
// each a CTA that builds the same table and probes a contiguous slice of the
// partition's S.
__global__ void k_units(PlanDev P) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= P.total_jparts) return;
    const uint32_t j = find_slot(P.jpart_prefix, P.njoin, t);
    const uint32_t p = t - P.jpart_prefix[j];
    uint32_t ns = 0, s0 = 0;
    const uint32_t g = unit_count_of(P, j, p, ns, s0);
    if (g == 0) return;
    JoinCtr *c = P.join[j].ctr;
    uint32_t first = 0;
    if (lane == 0) first = c->unit_base + atomicAdd(&c->unit_fill, g);
    first = __shfl_sync(0xffffffffu, first, 0);
    if (first + g > P.max_units) {
        if (lane == 0) atomicOr(&c->error, 4u);
        return;
    }
    for (uint32_t k = lane; k < g; k += 32) {
        Unit u;
        u.p = p;
        u.s_begin = s0 + (uint32_t)(((uint64_t)ns * k) / g);
        u.s_end = s0 + (uint32_t)(((uint64_t)ns * (k + 1)) / g);
        u.join = j;
        P.units[first + k] = u;
    }
}

// ------------------------------------------------------- output emission --
// The output state of the join a CTA is working on.
struct OutCtx {
    Tuple *out;
    uint32_t cap;  // plans keep the output below 2^32 pairs
    JoinCtr *ctr;
    uint32_t chunk;
};

__device__ __forceinline__ OutCtx out_ctx(const JoinDev &J) {
    OutCtx o;
    o.out = J.out;
    o.cap = (uint32_t)J.out_cap;
    o.ctr = J.ctr;
    o.chunk = J.out_chunk;
    return o;
}

struct WarpOut {
    uint32_t cur, end;  // output positions (below 2^32)
};

// Warp-aggregated append: one ballot per 32 candidate pairs; a fresh chunk of
// the join's output (out_chunk pairs, <= 1024) is reserved with one global
// atomic when the warp's chunk runs out.
__device__ __forceinline__ void warp_emit(const OutCtx &o, WarpOut &w, bool has, uint32_t lv, uint32_t rv) {
    const unsigned mask = __ballot_sync(0xffffffffu, has);
    if (mask == 0) return;
    const unsigned m = __popc(mask);
    const unsigned rank = __popc(mask & lanemask_lt());
    uint32_t pos;
    if (w.cur + m <= w.end) {
        pos = w.cur + rank;
        w.cur += m;
    } else {
        const uint32_t avail = w.end - w.cur;
        uint32_t nb = 0;
        if ((threadIdx.x & 31) == 0) {
            nb = (uint32_t)atomicAdd(&o.ctr->out_reserved, (unsigned long long)o.chunk);
            // a chunk beyond the capacity: its pairs are dropped and the join fails
            if (nb + o.chunk > o.cap) atomicOr(&o.ctr->error, 2u);
        }
        nb = __shfl_sync(0xffffffffu, nb, 0);
        pos = rank < avail ? w.cur + rank : nb + (rank - avail);
        w.cur = nb + (m - avail);
        w.end = nb + o.chunk;
    }
    if (has && pos < o.cap) reinterpret_cast<uint2 *>(o.out)[pos] = make_uint2(lv, rv);
}

// Records the unused tail of the warp's chunk as the warp's hole in join J.
__device__ __forceinline__ void warp_close(const JoinDev &J, WarpOut &w) {
    if ((threadIdx.x & 31) == 0 && w.end > w.cur) {
        const unsigned h = atomicAdd(&J.ctr->hole_count, 1u);
        if (h < kMaxHoles) {
            J.holes[h].begin = w.cur;
            J.holes[h].end = w.end;
        } else {
            atomicOr(&J.ctr->error, 8u);
        }
    }
    w.cur = w.end = 0u;
}

// Table slot of a key: Fibonacci (multiplicative) hashing -- the key times
// 2^32 / golden ratio, whose high bits are scaled to the table size
// (multiply-shift range reduction). Two multiplies; independent of the
// partition hash, so the keys of one partition spread over the whole table.
// (The reference's build hashes with its tabulation join_hash,
// a2a_srj_build.c:202-246; the slot function changes no result.)
__device__ __forceinline__ uint32_t slot_of(uint32_t key, uint32_t ts) {
    const uint32_t h = key * 0x9E3779B1u;
    return (uint32_t)(((unsigned long long)h * ts) >> 32);
}

// Clears the table and inserts the R partition. Linear probing, key 0 = empty
// (a2a_srj_build.c:208-246). A key already present is not inserted again, so the
// probe returns the first-inserted tuple of a repeated key, one match per S tuple
// (a2a_srj_probe_inner_mt.c:136-148).
__device__ __forceinline__ void build_table(const PlanDev &P, const JoinDev &J, uint32_t j, uint32_t p,
                                            unsigned long long *table) {
    const uint32_t ts = J.table_slots;  // even: cleared in 16-byte pairs
    ulonglong2 *t2 = reinterpret_cast<ulonglong2 *>(table);
    for (uint32_t i = threadIdx.x; i < ts / 2; i += blockDim.x) t2[i] = make_ulonglong2(0ull, 0ull);
    __syncthreads();
    const RelDev &Rr = P.rel[2 * j];
    const uint32_t nr = Rr.total[p];
    const Tuple *pr = Rr.out + Rr.base[p];
    constexpr int B = 4;  // loads in flight per thread
    for (uint32_t i0 = threadIdx.x; i0 < nr; i0 += B * blockDim.x) {
        Tuple t[B];
#pragma unroll
        for (int k = 0; k < B; k++) {
            const uint32_t i = i0 + k * blockDim.x;
            t[k] = i < nr ? pr[i] : Tuple{0u, 0u};
        }
#pragma unroll
        for (int k = 0; k < B; k++) {
            if (t[k].key == 0) continue;
            const unsigned long long ent = ((unsigned long long)t[k].pay << 32) | t[k].key;
            uint32_t s = slot_of(t[k].key, ts);
            for (uint32_t step = 0;; step++) {
                const unsigned long long prev = atomicCAS(&table[s], 0ull, ent);
                if (prev == 0ull || (uint32_t)prev == t[k].key) break;
                if (++s == ts) s = 0;
                if (step >= ts) {
                    atomicOr(&J.ctr->error, 1u);
                    break;
                }
            }
        }
    }
    __syncthreads();
}

// Probe of a2a_srj_probe_inner_mt.c:101-168: stop at the key (hit) or at an empty
// slot (miss). Slots are read in aligned pairs (one 16-byte shared load), which
// halves the steps of the linear scan; when the home slot s is odd, slot s-1 of
// the first pair lies before the probe sequence and is ignored. The first pair
// decides almost every probe at a load of 1/3: it is resolved with selects, and
// only a probe that finds both slots taken by other keys enters the loop. The
// scan is bounded by the table size. Key 0 (padding) must not hit: callers mask
// the result with key != 0 (its probe stops at the first empty slot).
__device__ __forceinline__ bool probe_table(const unsigned long long *table, uint32_t ts,
                                            uint32_t key, uint32_t &rpay) {
    const uint32_t s = slot_of(key, ts);
    const ulonglong2 *t2 = reinterpret_cast<const ulonglong2 *>(table);
    uint32_t p = s & ~1u;
    const ulonglong2 e = t2[p >> 1];
    const bool even = p == s;
    const uint32_t kx = (uint32_t)e.x, ky = (uint32_t)e.y;
    const bool hx = even && kx == key, ex = even && kx == 0;
    const bool hy = ky == key, ey = ky == 0;
    rpay = hx ? (uint32_t)(e.x >> 32) : (uint32_t)(e.y >> 32);
    if (hx || ex || hy || ey) return hx || (!ex && hy);
    p += 2;
    if (p >= ts) p = 0;
    for (uint32_t step = 1; step < ts / 2; step++) {
        const ulonglong2 f = t2[p >> 1];
        if ((uint32_t)f.x == key) {
            rpay = (uint32_t)(f.x >> 32);
            return true;
        }
        if ((uint32_t)f.x == 0) return false;
        if ((uint32_t)f.y == key) {
            rpay = (uint32_t)(f.y >> 32);
            return true;
        }
        if ((uint32_t)f.y == 0) return false;
        p += 2;
        if (p >= ts) p = 0;
    }
    return false;
}

// The unit range of local-join algorithm A (its units are contiguous in the queue).
__device__ __forceinline__ unsigned units_end(const PlanDev &P, int A) {
    return min(*(volatile unsigned *)&P.bctr->alg_begin[A + 1], P.max_units);
}

__device__ __forceinline__ unsigned claim_unit(const PlanDev &P, int A) {
    return *(volatile unsigned *)&P.bctr->alg_begin[A] + atomicAdd(&P.bctr->alg_next[A], 1u);
}

// Fetches the next unit of algorithm A for the CTA; false when its range is done.
__device__ __forceinline__ bool next_unit(const PlanDev &P, int A, unsigned n_units, unsigned *s_slot, Unit &un) {
    if (threadIdx.x == 0) *s_slot = claim_unit(P, A);
    __syncthreads();
    const unsigned u = *s_slot;
    __syncthreads();
    if (u >= n_units) return false;
    un = P.units[u];
    return true;
}

// Units claimed one ahead (the join kernels that build per partition): while
// a unit is probed, the CTA's last warp starts the next unit's R partition
// towards L2, so that unit's build finds its tuples there. unit_claim_first
// once, then unit_claim_next per unit; unit_prefetch_next_r after a barrier
// that follows unit_claim_next (the next index is written by thread 0).
__device__ __forceinline__ void unit_claim_first(const PlanDev &P, int A, unsigned *s_next) {
    if (threadIdx.x == 0) *s_next = claim_unit(P, A);
}

__device__ __forceinline__ bool unit_claim_next(const PlanDev &P, int A, unsigned n_units, unsigned *s_next,
                                                Unit &un) {
    __syncthreads();
    const unsigned u = *s_next;
    __syncthreads();
    if (u >= n_units) return false;
    un = P.units[u];
    if (threadIdx.x == 0) *s_next = claim_unit(P, A);
    return true;
}

__device__ __forceinline__ void unit_prefetch_next_r(const PlanDev &P, unsigned n_units, const unsigned *s_next,
                                                     const Unit &un) {
    if ((threadIdx.x >> 5) != (blockDim.x >> 5) - 1) return;
    const unsigned nu = *s_next;
    if (nu >= n_units) return;
    const Unit un2 = P.units[nu];
    if (un2.join == un.join && un2.p == un.p) return;  // the same table: nothing to fetch
    const RelDev &R2 = P.rel[2 * un2.join];
    const uint32_t nr2 = R2.total[un2.p];
    const Tuple *pr2 = R2.out + R2.base[un2.p];
    for (uint32_t i = (threadIdx.x & 31) * 16; i < nr2; i += 32 * 16) prefetch_l2(pr2 + i);
}

// Switches the CTA's output state to join j (closing the warp's chunk of the
// previous join, which leaves that join at most one hole per warp).
__device__ __forceinline__ void switch_join(const PlanDev &P, uint32_t j, uint32_t &cur_j, OutCtx &o, WarpOut &w) {
    if (j == cur_j) return;
    if (cur_j != 0xffffffffu) warp_close(P.join[cur_j], w);
    cur_j = j;
    o = out_ctx(P.join[j]);
}

// ----------------------------------------------------- partitioned hash join --
__global__ void __launch_bounds__(kJoinThreads, 2) k_join_phj(PlanDev P) {
    extern __shared__ unsigned long long table[];
    __shared__ unsigned s_next;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarps = kJoinThreads / 32;  // every join kernel runs kJoinThreads threads
    const unsigned n_units = units_end(P, SPJ_ALG_PHJ);
    WarpOut w{0u, 0u};
    OutCtx o{};
    uint32_t cur_j = 0xffffffffu, cur_p = 0xffffffffu;
    Unit un;
    unit_claim_first(P, SPJ_ALG_PHJ, &s_next);
    while (unit_claim_next(P, SPJ_ALG_PHJ, n_units, &s_next, un)) {
        const JoinDev &J = P.join[un.join];
        if (un.join != cur_j || un.p != cur_p) {
            switch_join(P, un.join, cur_j, o, w);
            build_table(P, J, un.join, un.p, table);
            cur_p = un.p;
        }
        else
            __syncthreads();  // the next unit's index is written
        unit_prefetch_next_r(P, n_units, &s_next, un);
        const uint32_t ts = J.table_slots;
        const Tuple *ps = P.rel[2 * un.join + 1].out;
        constexpr int U = 4;
        for (uint32_t base = un.s_begin + warp * 32 * U; base < un.s_end; base += nwarps * 32 * U) {
            // the warp's next 128 S tuples (8 lines) start towards L2 while these are probed
            const uint32_t nxt = base + nwarps * 32 * U + lane * 16;
            if (lane < 8 && nxt < un.s_end) prefetch_l2(ps + nxt);
            Tuple t[U];
            if (base + 32 * U <= un.s_end) {  // a whole step: no bounds per tuple
#pragma unroll
                for (int k = 0; k < U; k++) t[k] = ps[base + k * 32 + lane];
            } else {
#pragma unroll
                for (int k = 0; k < U; k++) {
                    const uint32_t idx = base + k * 32 + lane;
                    t[k] = idx < un.s_end ? ps[idx] : Tuple{0u, 0u};
                }
            }
#pragma unroll
            for (int k = 0; k < U; k++) {
                uint32_t rp = 0;
                const bool hit = probe_table(table, ts, t[k].key, rp) && t[k].key != 0;
                warp_emit(o, w, hit, rp, t[k].pay);
            }
        }
        __syncthreads();
    }
    if (cur_j != 0xffffffffu) warp_close(P.join[cur_j], w);
}

// Block-wide exclusive scan of n <= 1024 counters by warp 0 (8 per lane per
// step); writes off[0..n] (off[n] = total); callers synchronise.
__device__ __forceinline__ void warp0_scan1024(const uint32_t *cnt, uint32_t *off, int n) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    uint32_t carry = 0;
    for (int base = 0; base < n; base += 256) {  // 8 counters per lane per step
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int j = base + lane * 8 + i;
            c[i] = j < n ? cnt[j] : 0;
            sum += c[i];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        uint32_t run = carry + incl - sum;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int j = base + lane * 8 + i;
            if (j < n) off[j] = run;
            run += c[i];
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) off[n] = carry;
}

// ------------------------------------------------------------ sorted runs --
// The sort-merge join sorts every R partition once, before any work unit runs
// (mpsm_join_sort_probe.c:152-236 sorts each DPU's buckets once too), instead of
// once per unit: a hot partition split into hundreds of units was sorted
// hundreds of times. A partition of one unit is still sorted by that unit (a
// separate pass would only add a store and a load of its tuples). Runs of at
// most `cap` tuples (the largest power of two of the CTA's shared-memory budget)
// are sorted in place by (key, payload); a partition that fits is one run and is
// searched in shared memory, a larger one (many repeats of a key) is searched
// run by run in global memory. The nested-loop join, which sub-partitions its R
// partition in shared memory, takes the same run search for the partitions that
// do not fit.
__device__ __forceinline__ uint32_t run_cap(const JoinDev &J) {
    uint32_t cap = 1;
    while (cap * 2 <= (uint32_t)J.table_slots) cap <<= 1;
    return cap;
}

__device__ __forceinline__ unsigned long long pack_kp(const Tuple t) {
    return ((unsigned long long)t.key << 32) | t.pay;
}

// Bitonic sort of sorted[0, npad) (npad a power of two) by the whole CTA.
__device__ __forceinline__ void bitonic_sort_smem(unsigned long long *sorted, uint32_t npad) {
    for (uint32_t k = 2; k <= npad; k <<= 1) {
        for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
            for (uint32_t i = threadIdx.x; i < npad; i += blockDim.x) {
                const uint32_t ixj = i ^ jj;
                if (ixj > i) {
                    const unsigned long long a = sorted[i], b = sorted[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        sorted[i] = b;
                        sorted[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Whether k_sort_runs sorts R partition p of join j: a sort-merge partition
// with more than one work unit or beyond the shared-memory budget, a nested-loop
// partition beyond its budget.
__device__ __forceinline__ bool presorted(const PlanDev &P, uint32_t j, uint32_t p) {
    const JoinDev &J = P.join[j];
    const uint32_t nr = P.rel[2 * j].total[p];
    if (J.alg == SPJ_ALG_NL) return nr > (uint32_t)J.table_slots;
    if (J.alg != SPJ_ALG_SMJ) return false;
    if (nr > run_cap(J)) return true;
    uint32_t ns = 0, s0 = 0;
    return unit_count_of(P, j, p, ns, s0) > 1;
}

// Merge sort of a[0, npad) by the whole CTA with b[0, npad) as the second
// buffer (npad a power of two >= 8): runs of four sorted in registers, then
// log2(npad / 4) rounds in which every thread writes four outputs of a pair of
// runs, starting where the merge path (Odeh, Green, Mwassi, Shmueli, Birk,
// "Merge Path - Parallel Merging Made Simple", IPDPSW 2012) crosses its
// diagonal. Ten barriers for 4096 keys instead of the bitonic network's 78.
// Returns the buffer that holds the result.
__device__ __forceinline__ unsigned long long *merge_sort_smem(unsigned long long *a, unsigned long long *b,
                                                              uint32_t npad) {
    constexpr uint32_t E = 4;
    for (uint32_t g = threadIdx.x; g * E < npad; g += blockDim.x) {
        unsigned long long v0 = a[g * E], v1 = a[g * E + 1], v2 = a[g * E + 2], v3 = a[g * E + 3], t;
#define SPJ_CX(x, y) \
    if (x > y) {     \
        t = x;       \
        x = y;       \
        y = t;       \
    }
        SPJ_CX(v0, v1) SPJ_CX(v2, v3) SPJ_CX(v0, v2) SPJ_CX(v1, v3) SPJ_CX(v1, v2)
#undef SPJ_CX
        a[g * E] = v0;
        a[g * E + 1] = v1;
        a[g * E + 2] = v2;
        a[g * E + 3] = v3;
    }
    __syncthreads();
    unsigned long long *src = a, *dst = b;
    for (uint32_t L = E; L < npad; L <<= 1) {
        for (uint32_t k0 = threadIdx.x * E; k0 < npad; k0 += blockDim.x * E) {
            const uint32_t base = k0 & ~(2 * L - 1), d = k0 - base;
            const unsigned long long *A = src + base, *B = A + L;
            uint32_t lo = d > L ? d - L : 0, hi = min(d, L);
            while (lo < hi) {  // first i with A[i] > B[d - 1 - i]: ties take A first
                const uint32_t mid = (lo + hi) >> 1;
                if (A[mid] <= B[d - 1 - mid])
                    lo = mid + 1;
                else
                    hi = mid;
            }
            uint32_t i = lo, j = d - lo;
#pragma unroll
            for (uint32_t e = 0; e < E; e++) {
                const bool takeA = j >= L || (i < L && A[i] <= B[j]);
                dst[k0 + e] = takeA ? A[i++] : B[j++];
            }
        }
        __syncthreads();
        unsigned long long *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// Sorts buf[0, npad) (npad a power of two) by the whole CTA, using up to
// `room` entries of shared memory from buf; returns where the result is.
__device__ __forceinline__ unsigned long long *sort_smem(unsigned long long *buf, uint32_t npad, uint32_t room) {
    if (npad >= 8 && 2 * npad <= room) return merge_sort_smem(buf, buf + npad, npad);
    bitonic_sort_smem(buf, npad);
    return buf;
}

// Bucket sort by key range, the usual sort of an R run (<= 4096 tuples, four
// per thread): the run's smallest and largest key set the range, a counting pass
// drops every tuple into one of nb ~ n/2 buckets by (key - min) scaled to the
// range (monotone in the key: bucket order is key order), the buckets' offsets
// come from one scan, and each bucket (about two tuples) is put in (key, payload)
// order by one thread's insertion sort. The result is the same sequence as the
// merge sort's, from four barriers instead of ten rounds; hash partitioning
// spreads a partition's keys over their range, so buckets stay short. A bucket
// longer than kBucketMaxLen (many repeats of a key, or keys clustered in a
// small part of the range) makes the sort give up (nullptr, the same in every
// thread) and the caller merge-sorts; `a` is left unchanged.
constexpr uint32_t kBucketSortMax = 4096;  // tuples (four per thread of kJoinThreads)
constexpr uint32_t kBucketMaxLen = 32;
constexpr uint32_t kBucketsMax = 2048;

struct BucketSmem {
    uint32_t cnt[kBucketsMax + 1];  // bucket counts, then their exclusive offsets (cnt[nb] = n)
    uint32_t kmin, kmax, fail;
};

__device__ __forceinline__ unsigned long long *bucket_sort_smem(const unsigned long long *a, unsigned long long *b,
                                                               uint32_t n, BucketSmem &B) {
    constexpr int PER = kBucketSortMax / kJoinThreads;
    const int lane = threadIdx.x & 31;
    uint32_t nb = 32;
    while (nb < kBucketsMax && 2 * nb < n) nb <<= 1;
    if (threadIdx.x == 0) {
        B.kmin = 0xffffffffu;
        B.kmax = 0u;
        B.fail = 0u;
    }
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) B.cnt[i] = 0u;
    unsigned long long v[PER];
    uint32_t lo = 0xffffffffu, hi = 0u;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const uint32_t i = threadIdx.x + k * blockDim.x;
        v[k] = i < n ? a[i] : 0ull;
        if (i < n) {
            lo = min(lo, (uint32_t)(v[k] >> 32));
            hi = max(hi, (uint32_t)(v[k] >> 32));
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    __syncthreads();  // initial values written
    if (lane == 0) {
        atomicMin(&B.kmin, lo);
        atomicMax(&B.kmax, hi);
    }
    __syncthreads();
    const uint32_t kmin = B.kmin;
    const unsigned long long range = (unsigned long long)B.kmax - kmin + 1;  // >= 1 when n > 0
    // bucket = floor((key - kmin) * nb / range) < nb: exact when the range fits
    // the buckets, else a multiply-high by floor(2^32 * nb / range) (< 2^32)
    const bool direct = range <= nb;
    const uint32_t mult = direct ? 0u : (uint32_t)(((unsigned long long)nb << 32) / range);
    uint32_t br[PER];  // bucket << 16 | rank in the bucket
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const uint32_t i = threadIdx.x + k * blockDim.x;
        if (i < n) {
            const uint32_t d = (uint32_t)(v[k] >> 32) - kmin;
            const uint32_t bk = direct ? d : __umulhi(d, mult);
            br[k] = (bk << 16) | atomicAdd(&B.cnt[bk], 1u);
        }
    }
    __syncthreads();
    warp0_scan1024(B.cnt, B.cnt, (int)nb);  // in place: each lane reads its counters before writing them
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const uint32_t i = threadIdx.x + k * blockDim.x;
        if (i < n) b[B.cnt[br[k] >> 16] + (br[k] & 0xffffu)] = v[k];
    }
    __syncthreads();
    for (uint32_t bk = threadIdx.x; bk < nb; bk += blockDim.x) {
        const uint32_t s0 = B.cnt[bk], e0 = B.cnt[bk + 1];
        if (e0 - s0 > kBucketMaxLen) {
            B.fail = 1u;
        } else {
            for (uint32_t i = s0 + 1; i < e0; i++) {  // insertion sort of b[s0, e0)
                const unsigned long long x = b[i];
                uint32_t j = i;
                while (j > s0 && b[j - 1] > x) {
                    b[j] = b[j - 1];
                    j--;
                }
                b[j] = x;
            }
        }
    }
    __syncthreads();
    return B.fail ? nullptr : b;
}

// Sorts an R run: buf[0, n) holds it and buf[n, npad) padding (~0ull); `room`
// entries of shared memory from buf. Returns where the n sorted tuples are.
__device__ __forceinline__ const unsigned long long *sort_run_smem(unsigned long long *buf, uint32_t n, uint32_t npad,
                                                                   uint32_t room, BucketSmem &B) {
    if (n >= 64 && n <= kBucketSortMax && 2 * npad <= room) {
        const unsigned long long *r = bucket_sort_smem(buf, buf + npad, n, B);
        if (r) return r;
    }
    return sort_smem(buf, npad, room);
}

// One CTA per flat partition: the partitions `presorted` names, sorted in runs
// of run_cap tuples.
__global__ void __launch_bounds__(kJoinThreads, 2) k_sort_runs(PlanDev P) {
    extern __shared__ unsigned long long sorted[];
    __shared__ BucketSmem bsm;
    const uint32_t t = blockIdx.x;
    const uint32_t j = find_slot(P.jpart_prefix, P.njoin, t);
    const uint32_t p = t - P.jpart_prefix[j];
    const JoinDev &J = P.join[j];
    const RelDev &Rr = P.rel[2 * j];
    const uint32_t nr = Rr.total[p];
    if (nr == 0 || P.rel[2 * j + 1].total[p] == 0 || !presorted(P, j, p)) return;  // nothing to sort
    const uint32_t cap = run_cap(J);
    Tuple *pr = Rr.out + Rr.base[p];
    for (uint32_t r0 = 0; r0 < nr; r0 += cap) {
        const uint32_t len = min(cap, nr - r0);
        uint32_t npad = 1;
        while (npad < len) npad <<= 1;
        for (uint32_t i = threadIdx.x; i < npad; i += blockDim.x) sorted[i] = i < len ? pack_kp(pr[r0 + i]) : ~0ull;
        __syncthreads();
        const unsigned long long *res = sort_run_smem(sorted, len, npad, (uint32_t)J.table_slots, bsm);
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            const unsigned long long v = res[i];
            pr[r0 + i] = Tuple{(uint32_t)(v >> 32), (uint32_t)v};
        }
        __syncthreads();
    }
}

// The first tuple of key `key` in the sorted runs of pr[0, nr) (runs of cap
// tuples), read from global memory; false if none.
__device__ __forceinline__ bool search_runs(const Tuple *pr, uint32_t nr, uint32_t cap, uint32_t key, uint32_t &rp) {
    const unsigned long long target = (unsigned long long)key << 32;
    for (uint32_t r0 = 0; r0 < nr; r0 += cap) {
        uint32_t lo = r0, hi = min(nr, r0 + cap);
        const uint32_t end = hi;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (pack_kp(pr[mid]) < target)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo < end && pr[lo].key == key) {
            rp = pr[lo].pay;
            return true;
        }
    }
    return false;
}

// ---------------------------------------------------------- nested-loop join --
// nested_loop_join.c:184-231 on B200. The R partition is counting-sorted in
// shared memory into L <= 1024 sub-partitions (hash bits above the partition
// bits) of about 16 tuples on average (well under the 256 of the sweep's
// definition);
// each S tuple compares its key with every R tuple of its sub-partition and takes
// the first equal one. S is rewritten in place: unmatched S tuples are emitted
// unchanged.
__global__ void __launch_bounds__(kJoinThreads, 2) k_join_nl(PlanDev P) {
    extern __shared__ unsigned long long smem_u64[];
    __shared__ unsigned s_next;
    __shared__ uint32_t bcnt[1024], boff[1025];
    Tuple *rs = reinterpret_cast<Tuple *>(smem_u64);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarps = kJoinThreads / 32;  // every join kernel runs kJoinThreads threads
    const unsigned n_units = units_end(P, SPJ_ALG_NL);
    WarpOut w{0u, 0u};
    OutCtx o{};
    uint32_t cur_j = 0xffffffffu, cur_p = 0xffffffffu, nr = 0, lmask = 0;
    bool in_smem = true;
    const Tuple *pr_g = nullptr;
    Unit un;
    unit_claim_first(P, SPJ_ALG_NL, &s_next);
    while (unit_claim_next(P, SPJ_ALG_NL, n_units, &s_next, un)) {
        const JoinDev &J = P.join[un.join];
        const uint32_t bits = J.bits;
        if (un.join != cur_j || un.p != cur_p) {
            switch_join(P, un.join, cur_j, o, w);
            cur_p = un.p;
            const RelDev &Rr = P.rel[2 * un.join];
            const uint32_t cap = J.table_slots;  // R tuples that fit
            nr = Rr.total[un.p];
            pr_g = Rr.out + Rr.base[un.p];
            in_smem = nr <= cap;  // else: sorted runs, searched in global memory
            if (!in_smem) {
                __syncthreads();
                unit_prefetch_next_r(P, n_units, &s_next, un);
                goto probe;
            }
            uint32_t L = 1;
            while (L < 1024 && L * 16 < nr) L <<= 1;
            lmask = L - 1;
            for (uint32_t i = threadIdx.x; i < 1024; i += blockDim.x) bcnt[i] = 0;
            __syncthreads();
            const Tuple *pr = Rr.out + Rr.base[un.p];
            for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x)
                atomicAdd(&bcnt[(glb_partition_hash(pr[i].key) >> bits) & lmask], 1u);
            __syncthreads();
            warp0_scan1024(bcnt, boff, (int)L);
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) bcnt[i] = boff[i];
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) {
                const Tuple t = pr[i];
                const uint32_t b = (glb_partition_hash(t.key) >> bits) & lmask;
                rs[atomicAdd(&bcnt[b], 1u)] = t;
            }
            __syncthreads();
        } else {
            __syncthreads();  // the next unit's index is written
        }
        unit_prefetch_next_r(P, n_units, &s_next, un);
    probe:
        const Tuple *ps = P.rel[2 * un.join + 1].out;
        if (!in_smem) {  // an R partition beyond the shared-memory budget: its sorted runs
            const uint32_t rcap = run_cap(J);
            for (uint32_t base = un.s_begin + warp * 32; base < un.s_end; base += nwarps * 32) {
                const uint32_t idx = base + lane;
                const Tuple t = idx < un.s_end ? ps[idx] : Tuple{0u, 0u};
                uint32_t rp = 0;
                const bool hit = t.key != 0 && search_runs(pr_g, nr, rcap, t.key, rp);
                warp_emit(o, w, t.key != 0, hit ? rp : t.key, t.pay);
            }
            __syncthreads();
            continue;
        }
        constexpr int U = 4;
        for (uint32_t base = un.s_begin + warp * 32 * U; base < un.s_end; base += nwarps * 32 * U) {
            Tuple t[U];
#pragma unroll
            for (int k = 0; k < U; k++) {
                const uint32_t idx = base + k * 32 + lane;
                t[k] = idx < un.s_end ? ps[idx] : Tuple{0u, 0u};
            }
#pragma unroll
            for (int k = 0; k < U; k++) {
                const bool valid = t[k].key != 0;
                bool hit = false;
                uint32_t rp = 0;
                if (valid && nr) {
                    const uint32_t b = (glb_partition_hash(t[k].key) >> bits) & lmask;
                    for (uint32_t i = boff[b], e = boff[b + 1]; i < e; i++) {
                        const Tuple r = rs[i];
                        if (r.key == t[k].key) {
                            rp = r.pay;
                            hit = true;
                            break;
                        }
                    }
                }
                warp_emit(o, w, valid, hit ? rp : t[k].key, t[k].pay);
            }
        }
        __syncthreads();
    }
    if (cur_j != 0xffffffffu) warp_close(P.join[cur_j], w);
}

// ----------------------------------------------------------- sort-merge join --
// mpsm_join_sort_probe.c:152-236 on B200. The R partition, sorted once by
// k_sort_runs, is copied into shared memory, and every S tuple finds its key in
// it by a lower-bound search (the merge step of the reference, done per tuple:
// the output is a multiset, so S need not be sorted first -- sorting each warp's
// 32 S tuples with a shuffle network cost 30% of the join). A partition larger
// than the shared-memory budget is searched run by run in global memory. A
// matched S tuple becomes (R.payload, S.payload), an unmatched one stays as it
// is (S is rewritten in place).
__global__ void __launch_bounds__(kJoinThreads, 2) k_join_smj(PlanDev P) {
    extern __shared__ unsigned long long sorted[];
    __shared__ unsigned s_next;
    __shared__ BucketSmem bsm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarps = kJoinThreads / 32;  // every join kernel runs kJoinThreads threads
    const unsigned n_units = units_end(P, SPJ_ALG_SMJ);
    WarpOut w{0u, 0u};
    OutCtx o{};
    uint32_t cur_j = 0xffffffffu, cur_p = 0xffffffffu, nr = 0, cap = 1;
    bool in_smem = true;
    const Tuple *pr = nullptr;
    const unsigned long long *keys = sorted;  // the sorted partition in shared memory
    Unit un;
    unit_claim_first(P, SPJ_ALG_SMJ, &s_next);
    while (unit_claim_next(P, SPJ_ALG_SMJ, n_units, &s_next, un)) {
        const JoinDev &J = P.join[un.join];
        if (un.join != cur_j || un.p != cur_p) {
            switch_join(P, un.join, cur_j, o, w);
            cur_p = un.p;
            cap = run_cap(J);
            const RelDev &Rr = P.rel[2 * un.join];
            nr = Rr.total[un.p];
            pr = Rr.out + Rr.base[un.p];
            in_smem = nr <= cap;
            keys = sorted;
            if (in_smem && presorted(P, un.join, un.p)) {  // sorted once for all its units
                for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) sorted[i] = pack_kp(pr[i]);
            } else if (in_smem) {  // its only unit sorts it
                uint32_t npad = 1;
                while (npad < nr) npad <<= 1;
                for (uint32_t i = threadIdx.x; i < npad; i += blockDim.x) sorted[i] = i < nr ? pack_kp(pr[i]) : ~0ull;
                __syncthreads();
                keys = sort_run_smem(sorted, nr, npad, (uint32_t)J.table_slots, bsm);
            }
        }
        __syncthreads();  // the copy is complete and the next unit's index is written
        unit_prefetch_next_r(P, n_units, &s_next, un);
        const Tuple *ps = P.rel[2 * un.join + 1].out;
        for (uint32_t base = un.s_begin + warp * 32; base < un.s_end; base += nwarps * 32) {
            const uint32_t idx = base + lane;
            const bool in = idx < un.s_end;
            Tuple t = in ? ps[idx] : Tuple{0u, 0u};
            const bool valid = in && t.key != 0;
            bool hit = false;
            uint32_t rp = 0;
            if (valid && nr) {
                if (in_smem) {
                    const unsigned long long target = (unsigned long long)t.key << 32;
                    uint32_t lo = 0, hi = nr;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (keys[mid] < target)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    if (lo < nr && (uint32_t)(keys[lo] >> 32) == t.key) {
                        hit = true;
                        rp = (uint32_t)keys[lo];
                    }
                } else {
                    hit = search_runs(pr, nr, cap, t.key, rp);
                }
            }
            warp_emit(o, w, valid, hit ? rp : t.key, t.pay);
        }
        __syncthreads();
    }
    if (cur_j != 0xffffffffu) warp_close(P.join[cur_j], w);
}

// ------------------------------------------- non-partitioned hash join (NPHJ) --
// packetwise_no_partitioned_hash_join_build.c:88-160 / _probe.c:86-140 on B200:
// one linear-probe table per join over all of its R in HBM (2^k >= 2|R| slots,
// slot from join_hash2 as in the reference), built with 64-bit global CAS, then
// probed by a stream over S (units are raw S ranges). No partitioning pass; the
// table's random reads are served by L2 when R is small.
__global__ void k_nphj_clear(PlanDev P) {
    const JoinDev &J = P.join[blockIdx.y];
    if (J.alg != SPJ_ALG_NPHJ) return;
    ulonglong2 *t2 = reinterpret_cast<ulonglong2 *>(J.gtable);  // >= 1024 slots, a power of two
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < J.gtable_slots / 2;
         i += (unsigned long long)gridDim.x * blockDim.x)
        t2[i] = make_ulonglong2(0ull, 0ull);
}

// The build: one R tuple per thread and step, inserted into the join's
// linear-probing table by compare-and-swap (measured on B200 against four
// tuples per thread advanced together: 44.8 vs 56.9 us for 2^20 R tuples, 3.60
// vs 4.64 ms for 2^26).
__global__ void k_nphj_build(PlanDev P) {
    const uint32_t j = blockIdx.y;
    const JoinDev &J = P.join[j];
    if (J.alg != SPJ_ALG_NPHJ) return;
    const RelDev &Rr = P.rel[2 * j];
    const Tuple *r = Rr.in;
    const uint32_t n = Rr.n;
    const uint32_t tmask = (uint32_t)(J.gtable_slots - 1);
    unsigned long long *table = J.gtable;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Tuple t = r[i];
        if (t.key == 0 || !pred_pass(Rr.pred, t.key, t.pay)) continue;
        const unsigned long long ent = ((unsigned long long)t.pay << 32) | t.key;
        uint32_t s = join_hash2(t.key) & tmask;
        for (uint32_t step = 0; step <= tmask; step++) {
            const unsigned long long prev = atomicCAS(&table[s], 0ull, ent);
            if (prev == 0ull || (uint32_t)prev == t.key) break;
            s = (s + 1) & tmask;
            if (step == tmask) atomicOr(&J.ctr->error, 1u);
        }
    }
}


// Probes the U tuples t of a thread in the global table at once: every round
// resolves or advances each unresolved probe, so the thread waits for its
// longest probe sequence. Returns the mask of hits; e[k] is then the matching
// entry (R payload << 32 | key). Key-0 tuples (padding, not selected) miss.
template <int U>
__device__ __forceinline__ unsigned nphj_probe_all(const unsigned long long *table, uint32_t tmask, const Tuple (&t)[U],
                                                   unsigned long long (&e)[U]) {
    uint32_t sl[U];
    unsigned pend = 0, hit = 0;
#pragma unroll
    for (int k = 0; k < U; k++) {
        sl[k] = join_hash2(t[k].key) & tmask;
        e[k] = t[k].key ? __ldg(&table[sl[k]]) : 0ull;
        if (t[k].key) pend |= 1u << k;
    }
    for (uint32_t round = 0; pend && round <= tmask; round++) {
#pragma unroll
        for (int k = 0; k < U; k++) {
            if (!((pend >> k) & 1u)) continue;
            if ((uint32_t)e[k] == t[k].key) {
                hit |= 1u << k;
                pend &= ~(1u << k);
            } else if ((uint32_t)e[k] == 0u) {
                pend &= ~(1u << k);
            } else {
                sl[k] = (sl[k] + 1) & tmask;
            }
        }
#pragma unroll
        for (int k = 0; k < U; k++)
            if ((pend >> k) & 1u) e[k] = __ldg(&table[sl[k]]);
    }
    return hit;
}

// Probe of a non-partitioned join planned alone: CTAs stride over tiles of
// kJoinThreads * 4 S tuples with no work-unit list; each tile's pairs are
// counted per warp, the CTA reserves their space with one atomic and writes
// them densely, so the output has no holes and needs no fix-up. The last CTA to
// finish publishes the pair count (n_out and the caller's device counter).
// Pairs within the output are in no particular order (a join's output is a
// multiset); which R tuple of a repeated key matches is the first inserted, as
// in every hash join here.
__global__ void __launch_bounds__(kJoinThreads, 2) k_nphj_probe_direct(PlanDev P) {
    constexpr int U = 4, NW = kJoinThreads / 32;
    __shared__ uint32_t s_woff[NW];
    __shared__ uint32_t s_wcnt[NW];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const JoinDev &J = P.join[0];
    const RelDev &Rs = P.rel[1];
    const Tuple *s = Rs.in;
    const uint32_t n = Rs.n;
    const Pred pred = Rs.pred;
    const unsigned long long *table = J.gtable;
    const uint32_t tmask = (uint32_t)(J.gtable_slots - 1);
    uint2 *out = reinterpret_cast<uint2 *>(J.out);
    const unsigned long long cap = J.out_cap;
    JoinCtr *ctr = J.ctr;
    constexpr uint32_t T = kJoinThreads * U;
    for (uint32_t t0 = blockIdx.x * T; t0 < n; t0 += gridDim.x * T) {
        Tuple t[U];
        unsigned long long e[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const uint32_t idx = t0 + k * kJoinThreads + threadIdx.x;
            t[k] = idx < n ? s[idx] : Tuple{0u, 0u};
            if (t[k].key && !pred_pass(pred, t[k].key, t[k].pay)) t[k].key = 0;  // not selected
        }
        const unsigned hit = nphj_probe_all<U>(table, tmask, t, e);
        unsigned hits[U];
        uint32_t cnt = 0;
#pragma unroll
        for (int k = 0; k < U; k++) {
            hits[k] = __ballot_sync(0xffffffffu, (hit >> k) & 1u);
            cnt += __popc(hits[k]);
        }
        if (lane == 0) s_wcnt[warp] = cnt;
        __syncthreads();
        if (warp == 0) {
            const uint32_t c = s_wcnt[lane];
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
            }
            s_woff[lane] = incl - c;
            if (lane == 31) s_base = incl ? atomicAdd(&ctr->out_reserved, (unsigned long long)incl) : 0ull;
        }
        __syncthreads();
        unsigned long long pos = s_base + s_woff[warp];
#pragma unroll
        for (int k = 0; k < U; k++) {
            if ((hits[k] >> lane) & 1u) {
                const unsigned long long p = pos + __popc(hits[k] & lanemask_lt());
                if (p < cap)
                    out[p] = make_uint2((uint32_t)(e[k] >> 32), t[k].pay);
                else
                    atomicOr(&ctr->error, 2u);
            }
            pos += __popc(hits[k]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctr->probe_done, 1u) == gridDim.x - 1) {  // every other CTA has reserved its pairs
            __threadfence();
            const unsigned long long total = atomicAdd(&ctr->out_reserved, 0ull);
            const unsigned long long nout = total < cap ? total : cap;
            ctr->n_out = nout;
            if (J.n_out_user) *J.n_out_user = nout;
        }
    }
}

__global__ void __launch_bounds__(kJoinThreads, 2) k_nphj_probe(PlanDev P) {
    __shared__ unsigned s_slot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarps = kJoinThreads / 32;  // every join kernel runs kJoinThreads threads
    const unsigned n_units = units_end(P, SPJ_ALG_NPHJ);
    WarpOut w{0u, 0u};
    OutCtx o{};
    uint32_t cur_j = 0xffffffffu;
    Unit un;
    while (next_unit(P, SPJ_ALG_NPHJ, n_units, &s_slot, un)) {
        switch_join(P, un.join, cur_j, o, w);
        const JoinDev &J = P.join[un.join];
        const unsigned long long *table = J.gtable;
        const uint32_t tmask = (uint32_t)(J.gtable_slots - 1);
        const RelDev &Rs = P.rel[2 * un.join + 1];
        const Tuple *s = Rs.in;
        constexpr int U = 4;
        for (uint32_t base = un.s_begin + warp * 32 * U; base < un.s_end; base += nwarps * 32 * U) {
            Tuple t[U];
#pragma unroll
            for (int k = 0; k < U; k++) {
                const uint32_t idx = base + k * 32 + lane;
                t[k] = idx < un.s_end ? s[idx] : Tuple{0u, 0u};
                if (!pred_pass(Rs.pred, t[k].key, t[k].pay)) t[k].key = 0;  // not selected
            }
            uint32_t sl[U];
            unsigned long long e[U];
#pragma unroll
            for (int k = 0; k < U; k++) {
                sl[k] = join_hash2(t[k].key) & tmask;
                e[k] = t[k].key ? __ldg(&table[sl[k]]) : 0ull;
            }
#pragma unroll
            for (int k = 0; k < U; k++) {
                bool hit = false;
                uint32_t rp = 0;
                if (t[k].key) {
                    uint32_t sx = sl[k];
                    unsigned long long ex = e[k];
                    for (uint32_t step = 0; step <= tmask; step++) {
                        if ((uint32_t)ex == t[k].key) {
                            hit = true;
                            rp = (uint32_t)(ex >> 32);
                            break;
                        }
                        if ((uint32_t)ex == 0) break;
                        sx = (sx + 1) & tmask;
                        ex = __ldg(&table[sx]);
                    }
                }
                warp_emit(o, w, hit, rp, t[k].pay);
            }
        }
        __syncthreads();
    }
    if (cur_j != 0xffffffffu) warp_close(P.join[cur_j], w);
}

// ------------------------------------------------------------------ fix-up --
// Every reserved chunk is 1024-aligned and only a warp's last chunk of a join
// can be partly used, so the unused slots form at most one hole per warp and
// join, at a chunk's tail. With N = reserved - holes, the pairs stored at
// positions >= N outside holes move into the holes below N. One CTA per join.
// Exclusive scan in place of a[0..n) (n <= 13 * 1024) by a 1024-thread block;
// returns the total. Each thread scans 13 consecutive entries.
__device__ unsigned long long block_exclusive_scan(unsigned long long *a, unsigned n, unsigned long long *warp_tot) {
    constexpr int PER = 13;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned beg = threadIdx.x * PER;
    unsigned long long v[PER], sum = 0;
#pragma unroll
    for (int i = 0; i < PER; i++) {
        v[i] = beg + i < n ? a[beg + i] : 0ull;
        sum += v[i];
    }
    unsigned long long incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const unsigned long long w = warp_tot[lane];
        unsigned long long wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (unsigned)o) wi += t;
        }
        warp_tot[lane] = wi - w;
        if (lane == 31) warp_tot[32] = wi;
    }
    __syncthreads();
    unsigned long long run = warp_tot[warp] + incl - sum;
#pragma unroll
    for (int i = 0; i < PER; i++) {
        if (beg + i < n) a[beg + i] = run;
        run += v[i];
    }
    const unsigned long long total = warp_tot[32];
    __syncthreads();
    return total;
}

// Holes need no sort: each lies in its own chunk (a chunk's tail), so the holes
// at or above N are put in position order by indexing a slot array with their
// chunk number relative to N's chunk, and the gaps below N may be filled in
// any order (the output is a multiset). Three block scans per join.
__global__ void __launch_bounds__(1024) k_fixup_prep(PlanDev P) {
    extern __shared__ unsigned long long sm[];  // kUpSlots upper-hole slots, then kUpSlots scan slots
    unsigned long long *up = sm;                // (begin << 11) | length of the part above N, 0 = none
    unsigned long long *scan = sm + kUpSlots;
    __shared__ unsigned long long warp_tot[33];
    const JoinDev &J = P.join[blockIdx.x];
    JoinCtr *ctr = J.ctr;
    const unsigned nh = min(ctr->hole_count, (unsigned)kMaxHoles);
    const unsigned long long chunk = J.out_chunk;
    for (unsigned i = threadIdx.x; i < nh; i += blockDim.x) scan[i] = J.holes[i].end - J.holes[i].begin;
    __syncthreads();
    const unsigned long long H = block_exclusive_scan(scan, nh, warp_tot);
    const unsigned long long total = ctr->out_reserved;
    const unsigned long long N = total - H;
    const unsigned long long c0 = N / chunk;
    const unsigned long long ncu = total > N ? (total - 1) / chunk - c0 + 1 : 0;
    if (ncu > (unsigned long long)kUpSlots) {  // cannot happen while holes are chunk tails
        if (threadIdx.x == 0) atomicOr(&ctr->error, 8u);
        return;
    }
    for (unsigned k = threadIdx.x; k < ncu; k += blockDim.x) up[k] = 0ull;
    __syncthreads();
    // gap part (below N) of every hole, in hole order; upper part into its chunk's slot
    for (unsigned i = threadIdx.x; i < nh; i += blockDim.x) {
        const unsigned long long b = J.holes[i].begin, e = J.holes[i].end;
        scan[i] = b < N ? (e < N ? e : N) - b : 0ull;
        J.gaps[i].begin = b;
        if (e > N) {
            const unsigned long long ub = b > N ? b : N;
            up[ub / chunk - c0] = (ub << 11) | (e - ub);
        }
    }
    __syncthreads();
    const unsigned long long G = block_exclusive_scan(scan, nh, warp_tot);
    for (unsigned i = threadIdx.x; i < nh; i += blockDim.x) J.gap_off[i] = scan[i];
    __syncthreads();
    // upper holes in position order: their ranks, then the hole length before each
    for (unsigned k = threadIdx.x; k < ncu; k += blockDim.x) scan[k] = up[k] ? 1ull : 0ull;
    __syncthreads();
    const unsigned long long nd = block_exclusive_scan(scan, (unsigned)ncu, warp_tot);
    for (unsigned k = threadIdx.x; k < ncu; k += blockDim.x)
        if (up[k]) J.datas[scan[k]].end = k;  // slot of the rank-th upper hole
    __syncthreads();
    for (unsigned d = threadIdx.x; d < nd; d += blockDim.x) scan[d] = up[J.datas[d].end] & 2047ull;
    __syncthreads();
    block_exclusive_scan(scan, (unsigned)nd, warp_tot);
    for (unsigned d = threadIdx.x; d < nd; d += blockDim.x) {
        const unsigned long long u = up[J.datas[d].end];
        const unsigned long long ub = u >> 11;
        // data elements stored before this hole, and holes' length up to and including it
        J.datas[d].begin = ub - N - scan[d];
        J.data_off[d] = scan[d] + (u & 2047ull);
    }
    if (threadIdx.x == 0) {
        ctr->n_out = N;
        if (J.n_out_user) *J.n_out_user = N;
        ctr->gap_total = G;
        ctr->n_gaps = nh;
        ctr->n_data = (unsigned)nd;
    }
}

// One warp per gap (a hole below N): the gap's slots x in [gap_off, gap_off+len)
// of the "x-space" are filled from the pairs stored above N, in order; between
// consecutive upper holes the source is N + x + (length of the upper holes
// before it), so the warp finds its first data segment once and copies runs.
__global__ void k_fixup_copy(PlanDev P) {
    const JoinDev &J = P.join[blockIdx.y];
    JoinCtr *ctr = J.ctr;
    const unsigned long long G = ctr->gap_total;
    if (G == 0 || (ctr->error & 8u)) return;  // holes were dropped: the count is unusable
    const unsigned long long N = ctr->n_out;
    const unsigned ng = ctr->n_gaps, nd = ctr->n_data;
    uint2 *out = reinterpret_cast<uint2 *>(J.out);
    const int lane = threadIdx.x & 31;
    const unsigned wpb = blockDim.x >> 5;
    for (unsigned gi = blockIdx.x * wpb + (threadIdx.x >> 5); gi < ng; gi += gridDim.x * wpb) {
        const unsigned long long x0 = J.gap_off[gi];
        const unsigned long long x1 = gi + 1 < ng ? J.gap_off[gi + 1] : G;
        const unsigned long long d0 = J.gaps[gi].begin;
        // k = number of upper holes whose data prefix is <= x0
        unsigned lo = 0, hi = nd;
        while (lo < hi) {
            const unsigned mid = (lo + hi) >> 1;
            if (J.datas[mid].begin <= x0)
                lo = mid + 1;
            else
                hi = mid;
        }
        unsigned k = lo;
        unsigned long long x = x0;
        while (x < x1) {
            const unsigned long long shift = k > 0 ? J.data_off[k - 1] : 0ull;
            const unsigned long long brk = k < nd ? J.datas[k].begin : x1;
            const unsigned long long run_end = brk < x1 ? brk : x1;
            for (unsigned long long y = x + lane; y < run_end; y += 32) {
                const unsigned long long src = N + y + shift, dst = d0 + (y - x0);
                if (src >= J.out_cap || dst >= N)
                    atomicOr(&ctr->error, 16u);
                else
                    out[dst] = out[src];
            }
            x = run_end;
            k++;
        }
    }
}

// ------------------------------------------------------------- utilities --
__global__ void k_checksum(const spj_kv_pair_t *pairs, const int64_t *n_dev, unsigned long long *sum) {
    const unsigned long long n = (unsigned long long)*n_dev;
    unsigned long long acc = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        acc += pair_digest(pairs[i].lvalue, pairs[i].rvalue);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}

__global__ void k_gen_r(Perm pr, uint64_t n, Tuple *r) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        r[i] = gen_r(pr, i);
}

__global__ void k_gen_s(GenSpec g, Zipf z, Perm pr, Perm prank, Tuple *s, unsigned long long *expect) {
    unsigned long long acc = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < g.nS;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = gen_s_row(g, z, prank, j);
        Tuple t;
        t.key = (uint32_t)(1 + perm_apply(pr, row));
        t.pay = (uint32_t)j;
        s[j] = t;
        acc += pair_digest((uint32_t)row, (uint32_t)j);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (expect && (threadIdx.x & 31) == 0) atomicAdd(expect, acc);
}

// Selection: one CTA per 8192-tuple block; the block counts its selected
// tuples with ballots, reserves their range of the output with one atomic and
// writes them in input order (warp by warp, each warp's share placed by a scan
// of the warps' counts).
constexpr int kSelectBlock = 8192, kSelectThreads = 256;
__global__ void __launch_bounds__(kSelectThreads) k_select(const Tuple *in, uint64_t n, Pred pred, Tuple *out,
                                                            unsigned long long *n_out) {
    __shared__ uint32_t wcount[kSelectThreads / 32], wbase[kSelectThreads / 32];
    __shared__ unsigned long long s_base;
    constexpr int PER = kSelectBlock / kSelectThreads;  // 32 tuples per thread, warp-strided
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t b0 = (uint64_t)blockIdx.x * kSelectBlock; b0 < n; b0 += (uint64_t)gridDim.x * kSelectBlock) {
        // warp w covers [b0 + w * 1024, b0 + (w + 1) * 1024): 32 rounds of 32 tuples
        const uint64_t wb = b0 + (uint64_t)warp * (kSelectBlock / (kSelectThreads / 32));
        uint32_t masks[PER];
        uint32_t cnt = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint64_t i = wb + (uint64_t)k * 32 + lane;
            bool keep = false;
            if (i < n) {
                const Tuple t = in[i];
                keep = pred_pass(pred, t.key, t.pay);
            }
            masks[k] = __ballot_sync(0xffffffffu, keep);
            cnt += __popc(masks[k]);
        }
        if (lane == 0) wcount[warp] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int w = 0; w < kSelectThreads / 32; w++) {
                wbase[w] = run;
                run += wcount[w];
            }
            s_base = run ? atomicAdd(n_out, (unsigned long long)run) : 0ull;
        }
        __syncthreads();
        unsigned long long pos = s_base + wbase[warp];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint64_t i = wb + (uint64_t)k * 32 + lane;
            if ((masks[k] >> lane) & 1u) out[pos + __popc(masks[k] & lanemask_lt())] = in[i];
            pos += __popc(masks[k]);
        }
        __syncthreads();  // wcount / wbase / s_base are rewritten by the next block
    }
}

__global__ void k_hist_single(const Tuple *t, uint64_t n, int bits, uint32_t *hist) {
    const uint32_t mask = (1u << bits) - 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = t[i].key;
        if (k) atomicAdd(&hist[glb_partition_hash(k) & mask], 1u);
    }
}

}  // namespace spj

// Entry points used by spj_plan.cu and spj_noalloc.cu (C++ linkage, internal).
namespace spj {

cudaError_t init_single(spj_plan *pl, cudaStream_t st, bool keep_r) {
    const JoinHost &h = pl->joins[0];
    const uint32_t f = 1u << h.dev.bits;
    const uint32_t f1 = h.dev.fine_bits ? 1u << (h.dev.bits - h.dev.fine_bits) : 0u;
    static_assert((sizeof(BatchCtr) + sizeof(JoinCtr)) % 4 == 0, "counters in whole words");
    k_init_single<<<1, 32, 0, st>>>(pl->dev, h.rel[0], h.rel[1], h.dev, h.rel[0].nchunks, h.rel[1].nchunks, f, f1,
                                    keep_r && h.dev.alg != SPJ_ALG_NPHJ,
                                    (uint32_t)((sizeof(BatchCtr) + sizeof(JoinCtr)) / 4));
    return cudaGetLastError();
}

cudaError_t launch_pipeline(spj_plan *pl, cudaStream_t st, bool keep_r) {
    PlanDev P = pl->dev;
    const int M = P.alg_mask;
    const bool nphj = M & (1 << SPJ_ALG_NPHJ), part = M & ~(1 << SPJ_ALG_NPHJ);
    keep_r = keep_r && part;  // a non-partitioned join has no partitions to keep
    // a non-partitioned join alone whose table stays in L2 (<= 2^23 slots, the
    // planner's size) probes S directly: no work units, no fix-up. A larger
    // table's probes wait on HBM, where the direct probe's per-tile barriers
    // cost more than the units' warp-independent emission (C3 forced to the
    // non-partitioned join: 8.60 ms direct against 7.1 ms with units).
    const bool direct = nphj && !part && P.njoin == 1 && pl->joins[0].dev.gtable_slots <= (1ull << 23);
    if (keep_r) {
        // one-join plan whose R partitions (out, hist offsets, totals) are still in
        // its buffers from its previous execution: count and scatter S only. The
        // base scan still runs over both relations (it rederives R's bases and
        // largest partition from the kept totals).
        const JoinHost &h = pl->joins[0];
        P.total_chunks = h.rel[1].nchunks;
        P.total_parts = 1u << h.dev.bits;
        P.total_coarse = h.dev.fine_bits ? 1u << (h.dev.bits - h.dev.fine_bits) : 0u;
    }
    // timing events are recorded on eager launches only (not while a graph is captured)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    cudaEvent_t *ev = (pl->have_events && cap == cudaStreamCaptureStatusNone) ? pl->ring[pl->ring_next] : nullptr;
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], st);
    };
    const size_t jsm = (size_t)P.max_table_slots * 8;
    const uint32_t J = P.njoin;
    mark(0);
    if (part) {
        // heavy keys are sampled when R is partitioned; executions that keep R's
        // partitions keep its heavy table too
        if (P.any_heavy && !keep_r) k_heavy_sample<<<J, 1024, (size_t)kSampleSlots * 8, st>>>(P);
        k_hist<<<P.total_chunks, kHistThreads, ((size_t)4 << P.max_bits) + sizeof(HeavySmem), st>>>(P);
    }
    mark(1);
    if (part) {
        k_colscan<<<(P.total_parts + 255) / 256, 256, 0, st>>>(P);
        k_basescan<<<P.nrel, 1024, 0, st>>>(P);
    }
    mark(2);
    if (nphj) {  // the non-partitioned joins' global tables
        k_nphj_clear<<<dim3(pl->num_sms * 2, J), 256, 0, st>>>(P);
        k_nphj_build<<<dim3(pl->num_sms * 4, J), 256, 0, st>>>(P);
    }
    if (part) {
        k_scatter1<false><<<P.total_chunks, kScatterThreads, sizeof(TileSmem), st>>>(P);
        if (P.any_heavy)
            k_scatter1<true><<<P.total_chunks, kScatterThreads, sizeof(TileSmem) + sizeof(HeavySmem), st>>>(P);
        if (P.any_two_pass) {
            if (P.total_coarse) k_items<<<(P.total_coarse + 7) / 8, 256, 0, st>>>(P);
            k_scatter2<<<pl->num_sms * kScatterBlocksPerSM, kScatterThreads, sizeof(TileSmem), st>>>(P);
        }
        // R partitions searched by several sort-merge units (or too large for a
        // CTA) sorted once; also on executions that keep R's partitions, whose
        // units can differ from the previous execution's (sorting is idempotent)
        if (M & ((1 << SPJ_ALG_SMJ) | (1 << SPJ_ALG_NL))) k_sort_runs<<<P.total_jparts, kJoinThreads, jsm, st>>>(P);
    }
    mark(3);
    if (!direct) {
        k_units_count<<<(P.total_jparts + 255) / 256, 256, 0, st>>>(P);
        k_units_scan<<<1, 1024, 0, st>>>(P);
        k_units<<<(P.total_jparts * 32 + 255) / 256, 256, 0, st>>>(P);
    }
    mark(4);
    // one kernel per local-join algorithm in the plan, each over its own units
    if (M & (1 << SPJ_ALG_PHJ)) k_join_phj<<<pl->join_blocks, kJoinThreads, jsm, st>>>(P);
    if (M & (1 << SPJ_ALG_SMJ)) k_join_smj<<<pl->join_blocks, kJoinThreads, jsm, st>>>(P);
    if (M & (1 << SPJ_ALG_NL)) k_join_nl<<<pl->join_blocks, kJoinThreads, jsm, st>>>(P);
    if (direct)
        k_nphj_probe_direct<<<pl->join_blocks, kJoinThreads, 0, st>>>(P);
    else if (nphj)
        k_nphj_probe<<<pl->join_blocks, kJoinThreads, 0, st>>>(P);
    mark(5);
    if (!direct) {
        k_fixup_prep<<<J, 1024, (size_t)kUpSlots * 2 * 8, st>>>(P);
        // gaps are spread over all warps of a join's blocks; a batch gives each join fewer blocks
        k_fixup_copy<<<dim3(std::max<uint32_t>(64, (kMaxHoles + 7) / 8 / J), J), 256, 0, st>>>(P);
    }
    mark(6);
    if (ev) {
        pl->ring_next = (pl->ring_next + 1) % spj_plan::kRing;
        pl->ring_filled = pl->ring_filled < spj_plan::kRing ? pl->ring_filled + 1 : spj_plan::kRing;
    }
    return cudaGetLastError();
}

cudaError_t configure_kernels(int table_slots, int alg_mask, int *join_blocks_per_sm) {
    cudaError_t e;
    int dev = 0, max_smem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    e = cudaFuncSetAttribute(k_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (1 << kMaxRadixBits) * 4 + (int)sizeof(HeavySmem));
    if (e) return e;
    // the largest table any plan may use, so plans of different sizes coexist
    for (const void *k : {(const void *)k_join_phj, (const void *)k_join_smj, (const void *)k_join_nl,
                          (const void *)k_sort_runs}) {
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, k))) return e;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      max_smem - (int)fa.sharedSizeBytes - 1024)))
            return e;
    }
    e = cudaFuncSetAttribute(k_heavy_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, kSampleSlots * 8);
    if (e) return e;
    e = cudaFuncSetAttribute(k_scatter1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem));
    if (e) return e;
    e = cudaFuncSetAttribute(k_scatter1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(TileSmem) + sizeof(HeavySmem)));
    if (e) return e;
    e = cudaFuncSetAttribute(k_scatter2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem));
    if (e) return e;
    for (const void *k : {(const void *)k_scatter1<false>, (const void *)k_scatter1<true>, (const void *)k_scatter2, (const void *)k_join_phj,
                          (const void *)k_join_smj, (const void *)k_join_nl, (const void *)k_nphj_probe,
                          (const void *)k_hist})
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared)))
            return e;
    e = cudaFuncSetAttribute(k_fixup_prep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kUpSlots * 2 * 8);
    if (e) return e;
    const void *jk[4] = {(const void *)k_join_phj, (const void *)k_nphj_probe, (const void *)k_join_smj,
                         (const void *)k_join_nl};
    int best = 1 << 30;
    for (int a = 0; a < 4; a++) {
        if (!(alg_mask & (1 << a))) continue;
        int n = 0;
        const size_t dyn = a == SPJ_ALG_NPHJ ? 0 : (size_t)table_slots * 8;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, jk[a], kJoinThreads, dyn))) return e;
        best = std::min(best, n);
    }
    *join_blocks_per_sm = best == (1 << 30) ? 0 : best;
    return cudaSuccess;
}

cudaError_t launch_checksum(const spj_kv_pair_t *pairs, const int64_t *n_dev, uint64_t *sum_dev, int sms,
                            cudaStream_t st) {
    cudaMemsetAsync(sum_dev, 0, 8, st);
    k_checksum<<<sms * 4, 256, 0, st>>>(pairs, n_dev, reinterpret_cast<unsigned long long *>(sum_dev));
    return cudaGetLastError();
}

cudaError_t launch_generate(uint64_t seed, int64_t n_r, int64_t n_s, double zipf_s, spj_kv_pair_t *r,
                            spj_kv_pair_t *s, uint64_t *expect, int sms, cudaStream_t st) {
    const Perm pr = make_perm((uint64_t)n_r, seed_R(seed));
    const Perm prank = make_perm((uint64_t)n_r, seed_rank(seed));
    GenSpec g{seed, (uint64_t)n_r, (uint64_t)n_s, zipf_s};
    const Zipf z = make_zipf((uint64_t)n_r, zipf_s > 0 ? zipf_s : 1.0);
    if (expect) cudaMemsetAsync(expect, 0, 8, st);
    if (r && n_r > 0) k_gen_r<<<sms * 8, 256, 0, st>>>(pr, (uint64_t)n_r, reinterpret_cast<Tuple *>(r));
    if (s && n_s > 0)
        k_gen_s<<<sms * 8, 256, 0, st>>>(g, z, pr, prank, reinterpret_cast<Tuple *>(s),
                                          reinterpret_cast<unsigned long long *>(expect));
    return cudaGetLastError();
}

cudaError_t launch_select(const spj_kv_pair_t *in, int64_t n, const spj_predicate_t &p, spj_kv_pair_t *out,
                          int64_t *n_out, int sms, cudaStream_t st) {
    cudaMemsetAsync(n_out, 0, 8, st);
    if (n <= 0) return cudaGetLastError();
    const uint64_t blocks = std::min<uint64_t>(((uint64_t)n + kSelectBlock - 1) / kSelectBlock, (uint64_t)sms * 8);
    k_select<<<(unsigned)blocks, kSelectThreads, 0, st>>>(reinterpret_cast<const Tuple *>(in), (uint64_t)n,
                                                         Pred{(uint32_t)p.field, (uint32_t)p.op, p.lo, p.hi},
                                                         reinterpret_cast<Tuple *>(out),
                                                         reinterpret_cast<unsigned long long *>(n_out));
    return cudaGetLastError();
}

cudaError_t launch_hist_single(const spj_kv_pair_t *t, int64_t n, int bits, uint32_t *hist, int sms,
                               cudaStream_t st) {
    cudaMemsetAsync(hist, 0, (size_t)4 << bits, st);
    if (n > 0) k_hist_single<<<sms * 4, 256, 0, st>>>(reinterpret_cast<const Tuple *>(t), (uint64_t)n, bits, hist);
    return cudaGetLastError();
}

}  // namespace spj
