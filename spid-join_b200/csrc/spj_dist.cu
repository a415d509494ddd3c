// spj_dist.cu -- the join sharded over the GPUs of one node, driven from C.
//
// The reference shuffles every relation between its DPU ranks (the host's
// rotate-and-stream all-to-all, src/queryHostFunc.cc:481-777) and handles skew
// across ranks with rank sets: R is replicated to every rank group and S split
// among them (src/queryHostFunc.cc:654-776, glb_partition_count.c:317-318). Here
// every rank (one process per GPU) owns a shard of R and of S:
//
//   1. heavy keys: each rank samples its S and contributes its most frequent
//      keys; an all-gather gives every rank the same sorted list of the keys
//      whose estimated share of the global S is at least heavy_share / world;
//   2. the R tuples of heavy keys are all-gathered (replicated to every rank);
//      the S tuples of heavy keys stay on their rank;
//   3. every other tuple goes to rank (glb_partition_hash(key) * world) >> 32:
//      a device split groups the shard by destination (spj_exchange_split), an
//      all-gather shares the size matrix, and grouped NCCL sends and receives
//      move the groups over NVLink;
//   4. each rank joins what it received (plus the replicated heavy R tuples)
//      with its own plan; the union of the ranks' outputs is the join.
//
// NCCL is loaded when it is first needed (dlopen of libnccl.so.2), so the
// library itself does not depend on it; in a process that has loaded NCCL
// already (PyTorch does) the loader hands back that same library.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "spj_internal.h"

using namespace spj;

namespace {

// The NCCL entry points this file calls, resolved at run time.
struct Nccl {
    bool ok = false;
    std::string why;
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
    ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

Nccl &nccl() {
    static Nccl n;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            const char *e = dlerror();
            n.why = std::string("cannot load NCCL: ") + (e ? e : "libnccl.so.2 not found");
            return;
        }
        auto sym = [&](const char *name) {
            void *p = dlsym(h, name);
            if (!p && n.why.empty()) n.why = std::string("NCCL lacks ") + name;
            return p;
        };
        n.GetUniqueId = (decltype(n.GetUniqueId))sym("ncclGetUniqueId");
        n.CommInitRank = (decltype(n.CommInitRank))sym("ncclCommInitRank");
        n.CommDestroy = (decltype(n.CommDestroy))sym("ncclCommDestroy");
        n.CommAbort = (decltype(n.CommAbort))sym("ncclCommAbort");
        n.AllGather = (decltype(n.AllGather))sym("ncclAllGather");
        n.Send = (decltype(n.Send))sym("ncclSend");
        n.Recv = (decltype(n.Recv))sym("ncclRecv");
        n.GroupStart = (decltype(n.GroupStart))sym("ncclGroupStart");
        n.GroupEnd = (decltype(n.GroupEnd))sym("ncclGroupEnd");
        n.GetErrorString = (decltype(n.GetErrorString))sym("ncclGetErrorString");
        n.ok = n.why.empty();
    });
    return n;
}

int nccl_error(ncclResult_t r, const char *what) {
    return set_error(SPJ_E_CUDA, std::string(what) + ": " + nccl().GetErrorString(r));
}

#define SPJ_NCCL(call)                                       \
    do {                                                     \
        ncclResult_t r_ = (call);                            \
        if (r_ != ncclSuccess) return nccl_error(r_, #call); \
    } while (0)

#define SPJ_CUDA_D(call)                                     \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_error(e_, #call); \
    } while (0)

constexpr int kCand = 64;        // heavy-key candidates each rank contributes
constexpr int kMaxHeavyD = 256;  // heavy keys at most (the exchange kernels' limit)

// k keys of S at evenly spaced positions.
__global__ void k_dist_sample(const Tuple *s, uint64_t n, uint32_t k, uint32_t *keys) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint64_t idx = k > 1 ? (uint64_t)i * (n - 1) / (k - 1) : 0;
        keys[i] = s[idx].key;
    }
}

__device__ __forceinline__ bool in_sorted(const uint32_t *h, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (h[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < n && h[lo] == key;
}

// The R tuples of heavy keys, appended to out at an atomic cursor (at most cap).
__global__ void k_dist_heavy_rows(const Tuple *r, uint64_t n, const uint32_t *heavy, uint32_t nh, Tuple *out,
                                  unsigned long long *cnt, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const Tuple t = r[i];
        if (t.key && in_sorted(heavy, nh, t.key)) {
            const unsigned long long p = atomicAdd(cnt, 1ull);
            if (p < cap) out[p] = t;
        }
    }
}

// Gathered rows without their key-0 padding, compacted into out.
__global__ void k_dist_compact(const Tuple *in, uint64_t n, Tuple *out, unsigned long long *cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const Tuple t = in[i];
        if (t.key) out[atomicAdd(cnt, 1ull)] = t;
    }
}

// A device buffer that grows (stream-ordered) and is kept across calls.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int reserve(size_t need, cudaStream_t st) {
        if (need <= bytes) return SPJ_OK;
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
        const size_t b = std::max<size_t>(need + need / 4, 4096);
        cudaError_t e = cudaMallocAsync(&p, b, st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(sharded join buffer)");
        bytes = b;
        return SPJ_OK;
    }
    void release(cudaStream_t st) {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
    }
};

}  // namespace

struct spj_dist {
    ncclComm_t comm = nullptr;
    int world = 1, rank = 0;
    spj_design_t design{};
    double heavy_share = 0.25;
    int heavy_mode = 1;  // 0 off, 1 with more than one rank, 2 always
    uint32_t sample = 1u << 16;
    spj_plan_t *plan = nullptr;
    int64_t plan_r = -1, plan_s = -1;
    DevBuf keys, heavy, rows, rows_pad, rows_all, rows_cmp, grouped, recv_r, recv_s, cnt, cnt_all, out, misc;
    std::vector<uint32_t> last_heavy;
};

namespace {

// 1. The heavy keys, the same sorted list on every rank.
int dist_heavy_keys(spj_dist_t *d, const Tuple *s, int64_t n_s, cudaStream_t st, std::vector<uint32_t> &hot) {
    Nccl &N = nccl();
    hot.clear();
    const uint32_t k = (uint32_t)std::min<int64_t>(n_s, d->sample);
    std::vector<uint32_t> keys(k);
    int rc = d->keys.reserve((size_t)std::max<uint32_t>(k, 1) * 4, st);
    if (rc) return rc;
    if (k) {
        k_dist_sample<<<64, 256, 0, st>>>(s, (uint64_t)n_s, k, (uint32_t *)d->keys.p);
        SPJ_CUDA_D(cudaMemcpyAsync(keys.data(), d->keys.p, (size_t)k * 4, cudaMemcpyDeviceToHost, st));
        SPJ_CUDA_D(cudaStreamSynchronize(st));
    }
    std::unordered_map<uint32_t, uint64_t> freq;
    for (uint32_t key : keys)
        if (key) freq[key]++;
    std::vector<std::pair<uint64_t, uint32_t>> top;
    top.reserve(freq.size());
    for (auto &kv : freq) top.push_back({kv.second, kv.first});
    std::sort(top.begin(), top.end(), [](const std::pair<uint64_t, uint32_t> &a, const std::pair<uint64_t, uint32_t> &b) {
        return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    // (key, its estimated count in this rank's S) x kCand, then this rank's |S|
    const size_t per = 2 * kCand + 2;
    std::vector<unsigned long long> cand(per, 0ull);
    for (int i = 0; i < kCand && i < (int)top.size(); i++) {
        cand[2 * i] = top[i].second;
        cand[2 * i + 1] = (unsigned long long)((double)top[i].first * ((double)n_s / (double)std::max(k, 1u)));
    }
    cand[2 * kCand] = (unsigned long long)n_s;
    if ((rc = d->misc.reserve(per * 8 * (d->world + 1), st))) return rc;
    unsigned long long *dev = (unsigned long long *)d->misc.p;
    SPJ_CUDA_D(cudaMemcpyAsync(dev, cand.data(), per * 8, cudaMemcpyHostToDevice, st));
    SPJ_NCCL(N.AllGather(dev, dev + per, per, ncclUint64, d->comm, st));
    std::vector<unsigned long long> all(per * d->world);
    SPJ_CUDA_D(cudaMemcpyAsync(all.data(), dev + per, all.size() * 8, cudaMemcpyDeviceToHost, st));
    SPJ_CUDA_D(cudaStreamSynchronize(st));
    std::unordered_map<uint32_t, unsigned long long> est;
    unsigned long long total = 0;
    for (int w = 0; w < d->world; w++) {
        const unsigned long long *c = all.data() + per * w;
        for (int i = 0; i < kCand; i++)
            if (c[2 * i]) est[(uint32_t)c[2 * i]] += c[2 * i + 1];
        total += c[2 * kCand];
    }
    const double bar = d->heavy_share * (double)total / (double)d->world;
    std::vector<std::pair<unsigned long long, uint32_t>> h;
    for (auto &kv : est)
        if (kv.second > 0 && (double)kv.second >= bar) h.push_back({kv.second, kv.first});
    std::sort(h.begin(), h.end(),
              [](const std::pair<unsigned long long, uint32_t> &a, const std::pair<unsigned long long, uint32_t> &b) {
                  return a.first != b.first ? a.first > b.first : a.second < b.second;
              });
    for (int i = 0; i < kMaxHeavyD && i < (int)h.size(); i++) hot.push_back(h[i].second);
    std::sort(hot.begin(), hot.end());
    return SPJ_OK;
}

// 2. Every rank's R tuples of the heavy keys, compacted into d->rows_cmp on
// every rank; *n_rows = their number.
int dist_heavy_rows(spj_dist_t *d, const Tuple *r, int64_t n_r, const uint32_t *heavy_dev, int nh, int64_t *n_rows,
                    cudaStream_t st) {
    Nccl &N = nccl();
    int rc;
    if ((rc = d->rows.reserve((size_t)std::max<int64_t>(n_r, 1) * 8, st))) return rc;
    if ((rc = d->misc.reserve((size_t)(d->world + 2) * 8, st))) return rc;
    unsigned long long *c = (unsigned long long *)d->misc.p;
    SPJ_CUDA_D(cudaMemsetAsync(c, 0, 8, st));
    if (n_r > 0)
        k_dist_heavy_rows<<<256, 256, 0, st>>>(r, (uint64_t)n_r, heavy_dev, (uint32_t)nh, (Tuple *)d->rows.p, c,
                                              (uint64_t)n_r);
    SPJ_NCCL(N.AllGather(c, c + 1, 1, ncclUint64, d->comm, st));
    std::vector<unsigned long long> counts(d->world);
    SPJ_CUDA_D(cudaMemcpyAsync(counts.data(), c + 1, (size_t)d->world * 8, cudaMemcpyDeviceToHost, st));
    SPJ_CUDA_D(cudaStreamSynchronize(st));
    unsigned long long mx = 0, total = 0;
    for (auto v : counts) {
        mx = std::max(mx, v);
        total += v;
    }
    *n_rows = (int64_t)total;
    if (mx == 0) return SPJ_OK;
    // padded to the largest contribution with key-0 tuples, all-gathered, compacted
    if ((rc = d->rows_pad.reserve((size_t)mx * 8, st))) return rc;
    if ((rc = d->rows_all.reserve((size_t)mx * 8 * d->world, st))) return rc;
    if ((rc = d->rows_cmp.reserve((size_t)total * 8, st))) return rc;
    SPJ_CUDA_D(cudaMemsetAsync(d->rows_pad.p, 0, (size_t)mx * 8, st));
    const unsigned long long mine = counts[d->rank];
    if (mine) SPJ_CUDA_D(cudaMemcpyAsync(d->rows_pad.p, d->rows.p, (size_t)mine * 8, cudaMemcpyDeviceToDevice, st));
    SPJ_NCCL(N.AllGather(d->rows_pad.p, d->rows_all.p, (size_t)mx, ncclUint64, d->comm, st));
    SPJ_CUDA_D(cudaMemsetAsync(c, 0, 8, st));
    k_dist_compact<<<256, 256, 0, st>>>((const Tuple *)d->rows_all.p, (uint64_t)mx * d->world,
                                       (Tuple *)d->rows_cmp.p, c);
    return SPJ_OK;
}

// 3. All-to-all of one relation: split by destination, share the size matrix,
// move the groups; `extra` spare tuples after the received ones.
int dist_exchange(spj_dist_t *d, const Tuple *t, int64_t n, int mode, const uint32_t *heavy_dev, int nh,
                  DevBuf &recv, int64_t extra, int64_t *n_recv, cudaStream_t st) {
    Nccl &N = nccl();
    const int W = d->world;
    int rc;
    if ((rc = d->grouped.reserve((size_t)std::max<int64_t>(n, 1) * 8, st))) return rc;
    if ((rc = d->cnt.reserve((size_t)2 * W * 8, st))) return rc;
    if ((rc = d->cnt_all.reserve((size_t)W * W * 8, st))) return rc;
    const spj_kv_pair_t *src = n ? reinterpret_cast<const spj_kv_pair_t *>(t) : nullptr;
    rc = spj_exchange_split(src, n, W, d->rank, heavy_dev, nh, mode, (spj_kv_pair_t *)d->grouped.p,
                            (int64_t *)d->cnt.p, st);
    if (rc) return rc;
    SPJ_NCCL(N.AllGather(d->cnt.p, d->cnt_all.p, (size_t)W, ncclInt64, d->comm, st));
    std::vector<int64_t> m((size_t)W * W);
    SPJ_CUDA_D(cudaMemcpyAsync(m.data(), d->cnt_all.p, m.size() * 8, cudaMemcpyDeviceToHost, st));
    SPJ_CUDA_D(cudaStreamSynchronize(st));
    // m[src * W + dst]: the tuples rank src sends to rank dst
    int64_t got = 0;
    for (int w = 0; w < W; w++) got += m[(size_t)w * W + d->rank];
    if ((rc = recv.reserve((size_t)std::max<int64_t>(got + extra, 1) * 8, st))) return rc;
    Tuple *rb = (Tuple *)recv.p;
    const Tuple *gb = (const Tuple *)d->grouped.p;
    SPJ_NCCL(N.GroupStart());
    int64_t soff = 0, roff = 0;
    for (int w = 0; w < W; w++) {
        const int64_t sn = m[(size_t)d->rank * W + w], rn = m[(size_t)w * W + d->rank];
        if (sn) SPJ_NCCL(N.Send(gb + soff, (size_t)sn, ncclUint64, w, d->comm, st));
        if (rn) SPJ_NCCL(N.Recv(rb + roff, (size_t)rn, ncclUint64, w, d->comm, st));
        soff += sn;
        roff += rn;
    }
    SPJ_NCCL(N.GroupEnd());
    *n_recv = got;
    return SPJ_OK;
}

}  // namespace

extern "C" {

int spj_dist_unique_id(void *id_out) {
    if (!id_out) return set_error(SPJ_E_ARG, "NULL id buffer");
    Nccl &N = nccl();
    if (!N.ok) return set_error(SPJ_E_UNSUPPORTED, N.why);
    ncclUniqueId id;
    SPJ_NCCL(N.GetUniqueId(&id));
    memcpy(id_out, &id, sizeof(id));
    return SPJ_OK;
}

int spj_dist_create(const void *unique_id, int world, int rank, const spj_design_t *design, spj_dist_t **out) {
    if (!out || !unique_id || !design) return set_error(SPJ_E_ARG, "NULL argument");
    *out = nullptr;
    if (world < 1 || world > 1024 || rank < 0 || rank >= world) return set_error(SPJ_E_ARG, "bad world or rank");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(SPJ_E_NODEVICE, "no CUDA device available; libspidjoin has no CPU path");
    }
    Nccl &N = nccl();
    if (!N.ok) return set_error(SPJ_E_UNSUPPORTED, N.why);
    spj_dist_t *d = new spj_dist_t();
    d->world = world;
    d->rank = rank;
    d->design = *design;
    ncclUniqueId id;
    memcpy(&id, unique_id, sizeof(id));
    const ncclResult_t r = N.CommInitRank(&d->comm, world, id, rank);
    if (r != ncclSuccess) {
        delete d;
        return nccl_error(r, "ncclCommInitRank");
    }
    *out = d;
    return SPJ_OK;
}

int spj_dist_set_heavy(spj_dist_t *d, int mode, double share, int sample) {
    if (!d || mode < 0 || mode > 2 || !(share > 0) || sample < 1)
        return set_error(SPJ_E_ARG, "heavy keys: mode 0..2, share > 0, sample >= 1");
    d->heavy_mode = mode;
    d->heavy_share = share;
    d->sample = (uint32_t)sample;
    return SPJ_OK;
}

int spj_dist_join(spj_dist_t *d, const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s, int64_t n_s,
                  const spj_kv_pair_t **pairs, int64_t *n_pairs, void *stream) {
    if (!d || !pairs || !n_pairs || n_r < 0 || n_s < 0 || (n_r && !r) || (n_s && !s))
        return set_error(SPJ_E_ARG, "bad sharded-join arguments");
    if (!d->comm) return set_error(SPJ_E_STATE, "the communicator was aborted");
    if (((uintptr_t)r & 15) || ((uintptr_t)s & 15)) return set_error(SPJ_E_ARG, "shards must be 16-byte aligned");
    if (n_r >= kMaxTuples || n_s >= kMaxTuples) return set_error(SPJ_E_ARG, "shard sizes must stay below 2^32 - 2^24");
    cudaStream_t st = (cudaStream_t)stream;
    const Tuple *R = reinterpret_cast<const Tuple *>(r), *S = reinterpret_cast<const Tuple *>(s);
    int rc;
    // 1. heavy keys (every rank takes the same branches: the list is global)
    std::vector<uint32_t> hot;
    const bool use_heavy = d->heavy_mode == 2 || (d->heavy_mode == 1 && d->world > 1);
    if (use_heavy && (rc = dist_heavy_keys(d, S, n_s, st, hot))) return rc;
    d->last_heavy = hot;
    const int nh = (int)hot.size();
    if ((rc = d->heavy.reserve((size_t)std::max(nh, 1) * 4, st))) return rc;
    if (nh) SPJ_CUDA_D(cudaMemcpyAsync(d->heavy.p, hot.data(), (size_t)nh * 4, cudaMemcpyHostToDevice, st));
    const uint32_t *hd = (const uint32_t *)d->heavy.p;
    // 2. the replicated heavy R tuples, then 3. the exchanges: R (its heavy tuples
    // leave it) with room for the replicated rows after it, and S (heavy S stays)
    int64_t nrows = 0, nr = 0, ns = 0;
    if (nh && (rc = dist_heavy_rows(d, R, n_r, hd, nh, &nrows, st))) return rc;
    if ((rc = dist_exchange(d, R, n_r, nh ? 2 : 0, hd, nh, d->recv_r, nrows, &nr, st))) return rc;
    if ((rc = dist_exchange(d, S, n_s, nh ? 1 : 0, hd, nh, d->recv_s, 0, &ns, st))) return rc;
    if (nrows)
        SPJ_CUDA_D(cudaMemcpyAsync((Tuple *)d->recv_r.p + nr, d->rows_cmp.p, (size_t)nrows * 8,
                                   cudaMemcpyDeviceToDevice, st));
    // 4. the local join (its plan kept while the received sizes stay the same)
    const int64_t lr = nr + nrows, ls = ns;
    if (!d->plan || d->plan_r != lr || d->plan_s != ls) {
        if (d->plan) spj_plan_destroy(d->plan);
        d->plan = nullptr;
        if ((rc = spj_plan_create(lr, ls, &d->design, &d->plan))) return rc;
        d->plan_r = lr;
        d->plan_s = ls;
    }
    const int64_t cap = spj_plan_output_capacity(d->plan);
    if ((rc = d->out.reserve((size_t)cap * 8 + 16, st))) return rc;
    spj_kv_pair_t *outp = (spj_kv_pair_t *)d->out.p;
    int64_t *n_dev = (int64_t *)((char *)d->out.p + (size_t)cap * 8);
    // an empty relation still needs a readable, aligned column
    const spj_kv_pair_t *rj = lr ? (const spj_kv_pair_t *)d->recv_r.p : outp;
    const spj_kv_pair_t *sj = ls ? (const spj_kv_pair_t *)d->recv_s.p : outp;
    if ((rc = spj_plan_execute(d->plan, rj, sj, outp, n_dev, st))) return rc;
    int64_t n = 0;
    SPJ_CUDA_D(cudaMemcpyAsync(&n, n_dev, 8, cudaMemcpyDeviceToHost, st));
    SPJ_CUDA_D(cudaStreamSynchronize(st));
    spj_stats_t stats;
    if ((rc = spj_plan_stats(d->plan, &stats))) return rc;  // a device-side capacity check fired
    *pairs = outp;
    *n_pairs = n;
    return SPJ_OK;
}

int spj_dist_abort(spj_dist_t *d) {
    if (!d) return set_error(SPJ_E_ARG, "NULL handle");
    if (!d->comm) return SPJ_OK;  // aborted already
    const ncclResult_t r = nccl().CommAbort(d->comm);
    d->comm = nullptr;
    return r == ncclSuccess ? SPJ_OK : nccl_error(r, "ncclCommAbort");
}

int spj_dist_heavy_keys(const spj_dist_t *d, uint32_t *keys, int capacity) {
    if (!d) return 0;
    const int n = (int)d->last_heavy.size();
    if (keys)
        for (int i = 0; i < n && i < capacity; i++) keys[i] = d->last_heavy[i];
    return n;
}

void spj_dist_destroy(spj_dist_t *d) {
    if (!d) return;
    cudaDeviceSynchronize();
    for (DevBuf *b : {&d->keys, &d->heavy, &d->rows, &d->rows_pad, &d->rows_all, &d->rows_cmp, &d->grouped,
                      &d->recv_r, &d->recv_s, &d->cnt, &d->cnt_all, &d->out, &d->misc})
        b->release(0);
    if (d->plan) spj_plan_destroy(d->plan);
    if (d->comm) nccl().CommDestroy(d->comm);
    cudaDeviceSynchronize();
    delete d;
}

}  // extern "C"
