// spj_noalloc.cu -- the join for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at join time: a host runtime that has
// handed all of the GPU's memory to its own pool allocator, code that runs while
// a CUDA stream is being captured into a graph (allocation is not allowed in
// capture), or a real-time loop that must not block on the allocator. For them
// spj_join_noalloc runs the same partitioned hash join as spj_plan_execute, with
// every piece of scratch memory taken from one fixed region compiled into this
// library (kScratchBytes below), so the call itself allocates nothing. The price
// is a size limit (|R| <= 2^20, |S| <= 2^21) and one shared region: calls whose
// executions overlap on the GPU race on it.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "spj_internal.h"

namespace spj {

cudaError_t launch_pipeline(spj_plan *pl, cudaStream_t st);
cudaError_t configure_kernels(int table_slots, int alg, int *join_blocks_per_sm);

namespace {

constexpr int64_t kMaxR = 1ll << 20;
constexpr int64_t kMaxS = 1ll << 21;
constexpr size_t kScratchBytes = 32ull << 20;   // every GPU that loads the library holds this until exit
constexpr int kJoinBlocks = 64;                  // emitting CTAs: bounds the output slack below
constexpr int64_t kOutSlack = (int64_t)kJoinBlocks * (kJoinThreads / 32) * kOutChunk;  // = 2^21 pairs
constexpr int kMaxDevices = 64;

// The scratch region. Host code must not pass this symbol to a kernel: on the
// host it names a host-side stand-in, so its device address is looked up once
// per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct DeviceSetup {
    bool done = false;
    void *scratch = nullptr;
    int sms = 0;
    int table_slots_max = 0;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// One-time set-up on the current device: the scratch address and kernel
// attributes. Runs inside the first spj_join_noalloc call on that device.
int setup_device(int dev, DeviceSetup **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &s = g_setup[dev];
    if (!s.done) {
        cudaDeviceProp prop;
        cudaError_t e = cudaGetDeviceProperties(&prop, dev);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
        if (prop.major != 10)
            return set_error(SPJ_E_NODEVICE, std::string("libspidjoin is built for sm_100a; device is ") + prop.name);
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(scratch)");
        int max_smem = 0;
        e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return cuda_error(e, "cudaDeviceGetAttribute");
        int per_sm = 0;
        e = configure_kernels(kDefaultTableSlots, SPJ_ALG_PHJ, &per_sm);
        if (e != cudaSuccess) return cuda_error(e, "configure kernels");
        s.scratch = ptr;
        s.sms = prop.multiProcessorCount;
        s.table_slots_max = (max_smem - 1024) / 8;
        s.done = true;
    }
    *out = &s;
    return SPJ_OK;
}

// A negative count tells the caller that the join hit an internal capacity
// limit (the error bits are folded into the value): -1 - error.
__global__ void k_noalloc_status(const Counters *ctr, long long *n_out) {
    const unsigned err = ctr->error;
    if (err) *n_out = -1 - (long long)err;
}

int ceil_log2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) b++;
    return b;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace
}  // namespace spj

using namespace spj;

extern "C" int spj_join_noalloc(const spj_kv_pair_t *r, int64_t n_r, const spj_kv_pair_t *s, int64_t n_s,
                                spj_kv_pair_t *out, int64_t out_capacity, int64_t *n_out, void *stream) {
    if (n_r < 0 || n_s < 0 || n_r > kMaxR || n_s > kMaxS)
        return set_error(SPJ_E_ARG, "spj_join_noalloc takes |R| <= 2^20 and |S| <= 2^21 (its scratch is fixed); "
                                    "use spj_plan_create/spj_plan_execute for larger joins");
    if ((n_r && !r) || (n_s && !s) || !out || !n_out) return set_error(SPJ_E_ARG, "NULL column, output or count");
    if (((uintptr_t)r & 15) || ((uintptr_t)s & 15) || ((uintptr_t)out & 7) || ((uintptr_t)n_out & 7))
        return set_error(SPJ_E_ARG, "columns must be 16-byte aligned, output and count 8-byte aligned");
    if (out_capacity < n_s + kOutSlack)
        return set_error(SPJ_E_ARG, "spj_join_noalloc needs out_capacity >= |S| + 2^21 pairs");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(SPJ_E_NODEVICE, "device index out of range");
    DeviceSetup *ds = nullptr;
    int rc = setup_device(dev, &ds);
    if (rc) return rc;

    // The plan lives on the host stack; its device side points into the scratch.
    // One scatter pass (at most 256 partitions) keeps the scratch at two
    // partitioned columns plus small metadata.
    spj_plan pl;
    pl.n_r = n_r;
    pl.n_s = n_s;
    spj_design_default(&pl.design);
    pl.device = dev;
    pl.num_sms = ds->sms;
    pl.have_events = false;
    JoinParams &jp = pl.jp;
    jp.bits = std::min(std::max(ceil_log2((uint64_t)std::max<int64_t>(1, (n_r + 4095) / 4096)), 6), kMaxPassBits);
    jp.fine_bits = 0;
    {
        const double mean = (double)n_r / (double)(1ull << jp.bits);
        const int want = (int)std::max(1024.0, 3.0 * (mean + 6.0 * sqrt(mean) + 32.0));
        jp.table_slots = std::min((want + 255) / 256 * 256, ds->table_slots_max);
    }
    jp.alg = SPJ_ALG_PHJ;
    jp.skew_mode = SPJ_SKEW_ADAPTIVE;
    jp.group = 1;
    jp.unit_tuples = kDefaultUnitTuples;
    jp.keep_unmatched = 0;
    pl.join_blocks = kJoinBlocks;

    const int sms = ds->sms;
    const uint64_t F = 1ull << jp.bits;
    const int64_t ns[2] = {n_r, n_s};
    uint32_t nch[2], chunk[2];
    {
        int64_t c = std::max<int64_t>(4096, (n_r + n_s + 2 * sms - 3) / (2 * sms - 2));
        c = (c + 1) & ~1ll;
        for (int i = 0; i < 2; i++) {
            nch[i] = (uint32_t)std::max<int64_t>(1, (ns[i] + c - 1) / c);
            chunk[i] = (uint32_t)c;
        }
    }
    const uint64_t max_units = F + (uint64_t)n_s / jp.unit_tuples + F + 64;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    const size_t o_ctr = take(sizeof(Counters));
    const size_t o_hist0 = take((size_t)nch[0] * F * 4), o_hist1 = take((size_t)nch[1] * F * 4);
    const size_t o_tot0 = take(F * 4), o_tot1 = take(F * 4), o_base0 = take(F * 4), o_base1 = take(F * 4);
    const size_t o_pr = take((size_t)n_r * 8 + 16), o_ps = take((size_t)n_s * 8 + 16);
    const size_t o_units = take(max_units * sizeof(Unit));
    const size_t o_holes = take(kMaxHoles * sizeof(Hole));
    const size_t o_gaps = take(kMaxHoles * sizeof(Hole)), o_datas = take(kMaxHoles * sizeof(Hole));
    const size_t o_goff = take(kMaxHoles * 8), o_doff = take(kMaxHoles * 8);
    if (off > kScratchBytes) return set_error(SPJ_E_NOMEM, "scratch layout exceeds the fixed region");

    char *a = (char *)ds->scratch;
    PlanDev &P = pl.dev;
    memset(&P, 0, sizeof(P));
    P.ctr = (Counters *)(a + o_ctr);
    for (int i = 0; i < 2; i++) {
        P.rel[i].n = (uint32_t)ns[i];
        P.rel[i].chunk = chunk[i];
        P.rel[i].nchunks = nch[i];
        P.rel[i].tmp = nullptr;
        P.rel[i].chist = nullptr;
    }
    P.rel[0].in = reinterpret_cast<const Tuple *>(r);
    P.rel[1].in = reinterpret_cast<const Tuple *>(s);
    P.rel[0].hist = (uint32_t *)(a + o_hist0);
    P.rel[1].hist = (uint32_t *)(a + o_hist1);
    P.rel[0].total = (uint32_t *)(a + o_tot0);
    P.rel[1].total = (uint32_t *)(a + o_tot1);
    P.rel[0].base = (uint32_t *)(a + o_base0);
    P.rel[1].base = (uint32_t *)(a + o_base1);
    P.rel[0].out = (Tuple *)(a + o_pr);
    P.rel[1].out = (Tuple *)(a + o_ps);
    P.units = (Unit *)(a + o_units);
    P.max_units = (uint32_t)max_units;
    P.items = nullptr;
    P.max_items = 0;
    P.holes = (Hole *)(a + o_holes);
    P.gaps = (Hole *)(a + o_gaps);
    P.datas = (Hole *)(a + o_datas);
    P.gap_off = (unsigned long long *)(a + o_goff);
    P.data_off = (unsigned long long *)(a + o_doff);
    P.out = reinterpret_cast<Tuple *>(out);
    P.out_cap = (unsigned long long)out_capacity;
    P.n_out_user = reinterpret_cast<unsigned long long *>(n_out);
    // An empty relation still needs a readable, aligned column pointer.
    if (!P.rel[0].in) P.rel[0].in = P.rel[0].out;
    if (!P.rel[1].in) P.rel[1].in = P.rel[1].out;

    cudaStream_t st = (cudaStream_t)stream;
    // the region keeps the previous call's contents: the counters must start at zero
    e = cudaMemsetAsync(P.ctr, 0, sizeof(Counters), st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync(counters)");
    e = launch_pipeline(&pl, st);
    if (e != cudaSuccess) return cuda_error(e, "join kernels");
    k_noalloc_status<<<1, 1, 0, st>>>(P.ctr, reinterpret_cast<long long *>(n_out));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "status kernel");
    return SPJ_OK;
}
