// spj_noalloc.cu -- the join for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at join time: a database engine or other
// host runtime that has handed all of the GPU's memory to its own pool
// allocator (so a cudaMalloc from inside a query would fail or steal from the
// pool), or a latency-bound loop that must not stall on the allocator
// (cudaMalloc and cudaFree can synchronise the device). For them
// spj_join_noalloc runs the same partitioned hash join as spj_plan_execute, with
// every piece of scratch memory taken from one fixed region compiled into this
// library (kScratchBytes below), so the call itself allocates nothing. The price
// is a size limit (|R| <= 2^20, |S| <= 2^21) and one shared region: calls whose
// executions overlap on the GPU race on it. The first call on each device does
// a one-time set-up (the region's device address, kernel attributes); make that
// first call before capturing any stream.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "spj_internal.h"

namespace spj {

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
        e = configure_kernels(kDefaultTableSlots, 1 << SPJ_ALG_PHJ, &per_sm);
        if (e != cudaSuccess) return cuda_error(e, "configure kernels");
        s.scratch = ptr;
        s.sms = prop.multiProcessorCount;
        s.table_slots_max = max_table_slots_for(max_smem);
        s.done = true;
    }
    *out = &s;
    return SPJ_OK;
}

// A negative count tells the caller that the join hit an internal capacity
// limit (the error bits are folded into the value): -1 - error.
__global__ void k_noalloc_status(const JoinCtr *ctr, long long *n_out) {
    const unsigned err = ctr->error;
    if (err) *n_out = -1 - (long long)err;
}

int ceil_log2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) b++;
    return b;
}

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

    // The plan lives on the host; its device side points into the scratch. One
    // scatter pass (at most 256 partitions) keeps the scratch at two partitioned
    // columns plus small metadata.
    spj_plan pl;
    pl.n_r = n_r;
    pl.n_s = n_s;
    spj_design_default(&pl.design);
    pl.design.rank_num = 1;
    pl.design.heavy_sample = -1;  // no heavy-key table in the fixed region
    pl.device = dev;
    pl.num_sms = ds->sms;
    pl.have_events = false;
    pl.join_blocks = kJoinBlocks;
    pl.joins.resize(1);
    pl.shapes.resize(1);
    pl.joins[0].n_r = n_r;
    pl.joins[0].n_s = n_s;
    JoinShape sh = plan_shape(n_r, n_s, pl.design, ds->sms, ds->table_slots_max, true, 0, nullptr);
    sh.alg = SPJ_ALG_PHJ;  // the partitioned hash join (its scratch fits the fixed region)
    sh.gtable_slots = 0;
    sh.bits = std::min(std::max(ceil_log2((uint64_t)std::max<int64_t>(1, (n_r + 4095) / 4096)), 6), kMaxPassBits);
    sh.fine_bits = 0;
    {
        const double mean = (double)n_r / (double)(1ull << sh.bits);
        const int want = (int)std::max(1024.0, 3.0 * (mean + 6.0 * sqrt(mean) + 32.0));
        sh.table_slots = std::min((want + 255) / 256 * 256, ds->table_slots_max) & ~1;
    }
    sh.out_chunk = kOutChunk;
    pl.shapes[0] = sh;
    if (layout_plan(&pl, nullptr, false) > kScratchBytes)
        return set_error(SPJ_E_NOMEM, "scratch layout exceeds the fixed region");
    JoinHost &h = pl.joins[0];
    h.rel[0].in = reinterpret_cast<const Tuple *>(r);
    h.rel[1].in = reinterpret_cast<const Tuple *>(s);
    h.dev.out = reinterpret_cast<Tuple *>(out);
    h.dev.n_out_user = reinterpret_cast<unsigned long long *>(n_out);
    layout_plan(&pl, (char *)ds->scratch, false);
    h.dev.out_cap = (unsigned long long)out_capacity;
    // An empty relation still needs a readable, aligned column pointer.
    if (!h.rel[0].in) h.rel[0].in = h.rel[0].out;
    if (!h.rel[1].in) h.rel[1].in = h.rel[1].out;

    cudaStream_t st = (cudaStream_t)stream;
    // descriptors written by a kernel from its parameters (no host copy); the
    // same kernel zeroes the counters, which the region keeps from the last call
    e = init_single(&pl, st);
    if (e != cudaSuccess) return cuda_error(e, "descriptor kernel");
    e = launch_pipeline(&pl, st);
    if (e != cudaSuccess) return cuda_error(e, "join kernels");
    k_noalloc_status<<<1, 1, 0, st>>>(pl.dev.jctr, reinterpret_cast<long long *>(n_out));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "status kernel");
    return SPJ_OK;
}
