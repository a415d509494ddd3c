// spj_exchange.cu -- the split that precedes the rank-to-rank exchange of a
// join sharded over several GPUs.
//
// The reference shuffles every relation between its DPU ranks through the host
// (the rotate-and-stream all-to-all, src/queryHostFunc.cc:481-777, with
// destinations from the global partition hash, glb_partition_packet.c:420-464).
// Over NVLink the exchange is either one all-to-all per relation after each GPU
// has grouped its shard by destination rank (spj_exchange_split), or the split
// itself writing every tuple straight into its destination GPU's receive buffer
// through peer pointers (spj_exchange_scatter after spj_exchange_count): one
// kernel that partitions and sends, with no staging copy and no separate
// collective for the tuples. The destination of a key is glb_partition_hash(key)
// scaled to the number of ranks (multiply-shift), which leaves its low bits --
// the local partitions of the join that follows -- evenly spread on every rank.
#include <cuda_runtime.h>

#include "spj_internal.h"

using namespace spj;

namespace {

constexpr int kSplitThreads = 512;
constexpr int kSplitTile = 4096;  // tuples per block step
constexpr int kMaxWorld = 1024;

constexpr int kMaxHeavy = 256;
constexpr uint32_t kDrop = 0xffffffffu;

// Where a tuple goes. Heavy keys (SPID-Join's skew handling across ranks): the
// S tuples of a heavy key stay on their rank (keep_local) and the R tuples of a
// heavy key are replicated to every rank by the caller, so they leave this
// exchange (drop); other keys go to (glb_partition_hash(key) * world) >> 32.
struct Route {
    uint32_t world, me;
    int heavy_mode;  // 0: no heavy keys, 1: heavy stays on `me`, 2: heavy is dropped
    uint32_t nheavy;
    const uint32_t *heavy;  // sorted
};

__device__ __forceinline__ uint32_t dest_of(uint32_t key, uint32_t world) {
    return (uint32_t)(((unsigned long long)glb_partition_hash(key) * world) >> 32);
}

__device__ __forceinline__ uint32_t route_of(uint32_t key, const Route &rt, const uint32_t *heavy_sm) {
    if (rt.nheavy) {
        uint32_t lo = 0, hi = rt.nheavy;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (heavy_sm[mid] < key)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo < rt.nheavy && heavy_sm[lo] == key) return rt.heavy_mode == 1 ? rt.me : kDrop;
    }
    return dest_of(key, rt.world);
}

// Rank of the calling lane among the tuples of destination d in cnt[d]
// (cnt[d] += the group's size). With few destinations most lanes of a warp share
// one, so the lanes of a destination take consecutive ranks with one atomic per
// group (its stores then coalesce) instead of one serialised atomic each; with
// many destinations a plain atomic per lane is cheaper than the grouping.
// Called by the active lanes only (`act` = their mask).
__device__ __forceinline__ uint32_t rank_in(uint32_t *cnt, uint32_t d, unsigned act, bool grouped) {
    if (!grouped) return atomicAdd(&cnt[d], 1u);
    const unsigned peers = __match_any_sync(act, d);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cnt[d], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

constexpr uint32_t kGroupedWorld = 32;  // grouped ranking up to this many destinations

__device__ __forceinline__ void load_heavy(const Route &rt, uint32_t *heavy_sm) {
    for (uint32_t i = threadIdx.x; i < rt.nheavy; i += blockDim.x) heavy_sm[i] = rt.heavy[i];
}

// counts[d] += tuples of destination d (key-0 padding and dropped heavy keys
// are not counted).
__global__ void __launch_bounds__(kSplitThreads) k_split_count(const Tuple *in, unsigned long long n, Route rt,
                                                               unsigned long long *counts) {
    __shared__ uint32_t cnt[kMaxWorld];
    __shared__ uint32_t heavy_sm[kMaxHeavy];
    load_heavy(rt, heavy_sm);
    for (uint32_t d = threadIdx.x; d < rt.world; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const bool grouped = rt.world <= kGroupedWorld;
    // whole warps iterate together (the grouping needs the warp's lanes)
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i0 = (unsigned long long)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const unsigned long long i = i0 + threadIdx.x;
        const Tuple t = i < n ? in[i] : Tuple{0u, 0u};
        const uint32_t d = t.key ? route_of(t.key, rt, heavy_sm) : kDrop;
        const unsigned act = __ballot_sync(0xffffffffu, d != kDrop);
        if (d != kDrop) rank_in(cnt, d, act, grouped);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < rt.world; d += blockDim.x)
        if (cnt[d]) atomicAdd(&counts[d], (unsigned long long)cnt[d]);
}

// cursor[d] = exclusive prefix of counts (one warp; world <= 1024).
__global__ void k_split_offsets(const unsigned long long *counts, uint32_t world, unsigned long long *cursor) {
    const int lane = threadIdx.x;
    unsigned long long carry = 0;
    for (uint32_t base = 0; base < world; base += 32) {
        const uint32_t d = base + lane;
        const unsigned long long v = d < world ? counts[d] : 0ull;
        unsigned long long incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        if (d < world) cursor[d] = carry + incl - v;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// Each block step takes a tile, counts it per destination, reserves one range
// per destination with one atomic each and writes its tuples there, so a
// destination's tuples from one tile leave as one run. kPeers: destination d's
// tuples go to dests[d] (another GPU's receive buffer, written over NVLink);
// otherwise all go to `out`.
template <bool kPeers>
__global__ void __launch_bounds__(kSplitThreads) k_split_scatter(const Tuple *in, unsigned long long n, Route rt,
                                                                 unsigned long long *cursor, Tuple *out,
                                                                 Tuple *const *dests) {
    __shared__ uint32_t cnt[kMaxWorld];
    __shared__ unsigned long long base[kMaxWorld];
    __shared__ uint32_t heavy_sm[kMaxHeavy];
    const uint32_t world = rt.world;
    const bool grouped = world <= kGroupedWorld;
    constexpr int PER = kSplitTile / kSplitThreads;
    load_heavy(rt, heavy_sm);
    for (unsigned long long t0 = (unsigned long long)blockIdx.x * kSplitTile; t0 < n;
         t0 += (unsigned long long)gridDim.x * kSplitTile) {
        for (uint32_t d = threadIdx.x; d < world; d += blockDim.x) cnt[d] = 0;
        __syncthreads();
        Tuple v[PER];
        uint32_t dr[PER];  // destination << 16 | rank in the tile; 0xffffffff = none
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const unsigned long long i = t0 + threadIdx.x + (unsigned long long)k * kSplitThreads;
            v[k] = i < n ? in[i] : Tuple{0u, 0u};
            const uint32_t d = v[k].key ? route_of(v[k].key, rt, heavy_sm) : kDrop;
            const unsigned act = __ballot_sync(0xffffffffu, d != kDrop);
            dr[k] = d != kDrop ? (d << 16) | rank_in(cnt, d, act, grouped) : 0xffffffffu;
        }
        __syncthreads();
        for (uint32_t d = threadIdx.x; d < world; d += blockDim.x)
            base[d] = cnt[d] ? atomicAdd(&cursor[d], (unsigned long long)cnt[d]) : 0ull;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++)
            if (dr[k] != 0xffffffffu) {
                const uint32_t d = dr[k] >> 16;
                Tuple *dst = kPeers ? dests[d] : out;
                dst[base[d] + (dr[k] & 0xffffu)] = v[k];
            }
        __syncthreads();
    }
}

}  // namespace

static int exchange_device(int *sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    return SPJ_OK;
}

static int make_route(int world, int me, const uint32_t *heavy, int n_heavy, int heavy_mode, Route *rt) {
    if (world < 1 || world > kMaxWorld) return set_error(SPJ_E_ARG, "world must be in [1, 1024]");
    if (me < 0 || me >= world) return set_error(SPJ_E_ARG, "rank outside the world");
    if (n_heavy < 0 || n_heavy > kMaxHeavy || (n_heavy > 0 && !heavy) || heavy_mode < 0 || heavy_mode > 2)
        return set_error(SPJ_E_ARG, "heavy keys: at most 256, sorted, mode 0..2");
    *rt = Route{(uint32_t)world, (uint32_t)me, heavy_mode, heavy_mode ? (uint32_t)n_heavy : 0u, heavy};
    return SPJ_OK;
}

extern "C" {

int spj_exchange_split(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                       int n_heavy, int heavy_mode, spj_kv_pair_t *out, int64_t *counts, void *stream) {
    Route rt;
    int rc = make_route(world, me, heavy_keys, n_heavy, heavy_mode, &rt);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!tuples || !out)) || !counts) return set_error(SPJ_E_ARG, "bad split arguments");
    int sms = 0;
    if ((rc = exchange_device(&sms))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(counts);
    unsigned long long *cursor = cnt + world;
    cudaError_t e = cudaMemsetAsync(cnt, 0, (size_t)world * 8, st);
    if (e != cudaSuccess) return cuda_error(e, "split counters");
    const Tuple *in = reinterpret_cast<const Tuple *>(tuples);
    if (n > 0) k_split_count<<<sms * 4, kSplitThreads, 0, st>>>(in, (unsigned long long)n, rt, cnt);
    k_split_offsets<<<1, 32, 0, st>>>(cnt, (uint32_t)world, cursor);
    if (n > 0)
        k_split_scatter<false><<<sms * 4, kSplitThreads, 0, st>>>(in, (unsigned long long)n, rt, cursor,
                                                                   reinterpret_cast<Tuple *>(out), nullptr);
    e = cudaGetLastError();
    return e ? cuda_error(e, "split kernels") : SPJ_OK;
}

int spj_exchange_count(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                       int n_heavy, int heavy_mode, int64_t *counts, void *stream) {
    Route rt;
    int rc = make_route(world, me, heavy_keys, n_heavy, heavy_mode, &rt);
    if (rc) return rc;
    if (n < 0 || (n > 0 && !tuples) || !counts) return set_error(SPJ_E_ARG, "bad count arguments");
    int sms = 0;
    if ((rc = exchange_device(&sms))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counts, 0, (size_t)world * 8, st);
    if (e == cudaSuccess && n > 0)
        k_split_count<<<sms * 4, kSplitThreads, 0, st>>>(reinterpret_cast<const Tuple *>(tuples),
                                                         (unsigned long long)n, rt,
                                                         reinterpret_cast<unsigned long long *>(counts));
    if (e == cudaSuccess) e = cudaGetLastError();
    return e ? cuda_error(e, "count kernel") : SPJ_OK;
}

int spj_exchange_scatter(const spj_kv_pair_t *tuples, int64_t n, int world, int me, const uint32_t *heavy_keys,
                         int n_heavy, int heavy_mode, spj_kv_pair_t *const *dest_bufs, const int64_t *dest_offsets,
                         int64_t *cursor, void *stream) {
    Route rt;
    int rc = make_route(world, me, heavy_keys, n_heavy, heavy_mode, &rt);
    if (rc) return rc;
    if (n < 0 || (n > 0 && !tuples) || !dest_bufs || !dest_offsets || !cursor)
        return set_error(SPJ_E_ARG, "bad scatter arguments");
    int sms = 0;
    if ((rc = exchange_device(&sms))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(cursor, dest_offsets, (size_t)world * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && n > 0)
        k_split_scatter<true><<<sms * 4, kSplitThreads, 0, st>>>(
            reinterpret_cast<const Tuple *>(tuples), (unsigned long long)n, rt,
            reinterpret_cast<unsigned long long *>(cursor), nullptr, reinterpret_cast<Tuple *const *>(dest_bufs));
    if (e == cudaSuccess) e = cudaGetLastError();
    return e ? cuda_error(e, "exchange scatter kernel") : SPJ_OK;
}

}  // extern "C"
