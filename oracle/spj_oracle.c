/*
 * spj_oracle.c -- CPU restatement of SPID-Join's equi-join path: the ORACLE.
 *
 * This file is test infrastructure. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline legs of bench.py load it, and only as the checker or as the timed
 * CPU baseline. The product library (libspidjoin) never links or calls it.
 *
 * Everything here follows the reference project yonsei-hpcp/spid-join; paths below
 * are relative to that project's root:
 *
 *   hashes ................ src/dpu/src/hash.c:15-178 (CRC table, join_hash,
 *                           join_hash2, glb_partition_hash, local_partition_hash)
 *   column split .......... src/query.cc:213-317 (JoinInstance::LoadColumn)
 *   global count (R, S) ... src/dpu/src/join/glb_partition_count.c:119-371
 *   R replication ......... src/queryHostFunc.cc:654-776 (rankgroup_aware RNS)
 *   bank-set R broadcast .. src/dpu/src/join/bg_broadcast_count.c:119-259,
 *                           src/queryHostFunc.cc:1181-1419
 *   chip-wise S split ..... src/dpu/src/join/glb_chipwise_partition_count.c:132-139,251-255
 *   local partitioning .... src/dpu/src/join/a2a_packetwise_srj_local_partition.c:142-228,323-350
 *                           (S reuses R's count: src/queryCompoundFunc.cc:103-122)
 *   hash build ............ src/dpu/src/join/a2a_srj_build.c:202-296
 *   hash probe ............ src/dpu/src/join/a2a_srj_probe_inner_mt.c:101-168
 *   sort-merge ............ src/dpu/src/join/mpsm_join_sort_probe.c:152-236
 *                           (range buckets: mpsm_join_local_partition.c:137,203-207)
 *   nested loop ........... src/dpu/src/join/nested_loop_join.c:184-231
 *   non-partitioned hash .. src/dpu/src/join/packetwise_no_partitioned_hash_join_build.c:101-166,
 *                           packetwise_no_partitioned_hash_join_probe.c:65-160 (one table over
 *                           the DPU's R, first match per S tuple: the pairs of the hash join
 *                           above, which the refpipe join runs for it)
 *
 * The CRC table is generated from the reflected CRC-32 polynomial 0xEDB88320; the
 * reference ships the same table literally (hash.c:15-59). The test suite pins
 * every hash here against the reference's own hash.c compiled from source
 * (oracle/Makefile target `ref`).
 *
 * Tuples are the reference's kv_pair_t / tuplePair_t: {u32 lvalue = key,
 * u32 rvalue = payload}; key 0 marks an empty slot or padding and never joins.
 * Output pairs are {lvalue = R payload, rvalue = S payload}; for the sort-merge
 * and nested-loop algorithms an S tuple without a match is emitted unchanged
 * (its key stays in lvalue), as those kernels rewrite S in place.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <math.h>

typedef struct { uint32_t key, pay; } orc_tuple;

enum {
    ORC_OK = 0,
    ORC_E_ARG = -1,
    ORC_E_NOMEM = -2,
    ORC_E_TABLE_FULL = -3,   /* a local partition holds more than 4096 R tuples */
};

enum { ORC_ALG_PHJ = 0, ORC_ALG_NPHJ = 1, ORC_ALG_SMJ = 2, ORC_ALG_NL = 3 };

/* ---------------------------------------------------------------- hashes -- */

static uint32_t g_crc[256];
static pthread_once_t g_crc_once = PTHREAD_ONCE_INIT;

static void crc_init(void)
{
    for (uint32_t i = 0; i < 256; i++) {
        uint32_t c = i;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
        g_crc[i] = c;
    }
}

static const uint32_t *crc(void)
{
    pthread_once(&g_crc_once, crc_init);
    return g_crc;
}

const uint32_t *orc_crc_table(void) { return crc(); }

/* hash.c:72-83. In C, & binds tighter than ^, so only byte 0 is masked. */
uint32_t orc_join_hash(uint32_t key)
{
    const uint32_t *t = crc();
    return (0xd9d65adcu & t[key & 0xffu]) ^ t[(key >> 8) & 0xffu] ^ t[(key >> 16) & 0xffu] ^
           t[(key >> 24) & 0xffu];
}

/* hash.c:85-112: Jenkins one-at-a-time over the four little-endian key bytes. */
uint32_t orc_join_hash2(uint32_t key)
{
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

/* hash.c:117-166: SuperFastHash-style over 4 bytes, seed = length = 4. The main
 * loop runs once (len>>2 == 1) and there is no tail (len&3 == 0). */
uint32_t orc_glb_partition_hash(uint32_t key)
{
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

/* hash.c:168-178: tabulation of key>>6 with byte 0 masked by 0xbfd06116. */
uint32_t orc_local_partition_hash(uint32_t key)
{
    const uint32_t *t = crc();
    uint32_t k = key >> 6;
    return (0xbfd06116u & t[k & 0xffu]) ^ t[(k >> 8) & 0xffu] ^ t[(k >> 16) & 0xffu] ^
           t[(k >> 24) & 0xffu];
}

/* splitmix64 finaliser (Steele, Lea, Flood 2014); the order-independent checksum
 * of an output multiset is the wrapping sum of mix64((u64)lvalue<<32 | rvalue). */
static inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

uint64_t orc_checksum(const orc_tuple *p, int64_t n)
{
    uint64_t s = 0;
    for (int64_t i = 0; i < n; i++) s += mix64(((uint64_t)p[i].key << 32) | p[i].pay);
    return s;
}

/* Canonical order: ascending (lvalue, rvalue). LSD radix sort, 4 x 16-bit digits. */
int orc_sort_pairs(orc_tuple *p, int64_t n)
{
    if (n <= 1) return ORC_OK;
    uint64_t *a = (uint64_t *)malloc((size_t)n * 8), *b = (uint64_t *)malloc((size_t)n * 8);
    int64_t *cnt = (int64_t *)malloc(65536 * sizeof(int64_t));
    if (!a || !b || !cnt) { free(a); free(b); free(cnt); return ORC_E_NOMEM; }
    for (int64_t i = 0; i < n; i++) a[i] = ((uint64_t)p[i].key << 32) | p[i].pay;
    for (int pass = 0; pass < 4; pass++) {
        int sh = 16 * pass;
        memset(cnt, 0, 65536 * sizeof(int64_t));
        for (int64_t i = 0; i < n; i++) cnt[(a[i] >> sh) & 0xffff]++;
        int64_t run = 0;
        for (int d = 0; d < 65536; d++) { int64_t c = cnt[d]; cnt[d] = run; run += c; }
        for (int64_t i = 0; i < n; i++) b[cnt[(a[i] >> sh) & 0xffff]++] = a[i];
        uint64_t *t = a; a = b; b = t;
    }
    for (int64_t i = 0; i < n; i++) { p[i].key = (uint32_t)(a[i] >> 32); p[i].pay = (uint32_t)a[i]; }
    free(a); free(b); free(cnt);
    return ORC_OK;
}

/* ----------------------------------------------------------- thread pool -- */

typedef void (*task_fn)(void *ctx, int64_t i);
typedef struct { task_fn fn; void *ctx; int64_t n; int64_t next; } pfor_t;

static void *pfor_worker(void *arg)
{
    pfor_t *pf = (pfor_t *)arg;
    for (;;) {
        int64_t i = __atomic_fetch_add(&pf->next, 1, __ATOMIC_RELAXED);
        if (i >= pf->n) break;
        pf->fn(pf->ctx, i);
    }
    return NULL;
}

static void parallel_for(int nthreads, int64_t n, task_fn fn, void *ctx)
{
    pfor_t pf = {fn, ctx, n, 0};
    if (nthreads <= 1 || n <= 1) { pfor_worker(&pf); return; }
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; t++)
        if (pthread_create(&th[started], NULL, pfor_worker, &pf) == 0) started++;
    pfor_worker(&pf);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------- global partition count -- */

/* glb_partition_count.c:119-371 over ONE source block (one DPU's input).
 * type 0 (R): id = h & (P-1).
 * type 1 (S): id = (h & (P/rank_sets - 1)) + (i & (rank_sets-1)) * ranks_per_set*64,
 *             where i is the tuple's index inside its 2048-byte read block
 *             (ELEM_PER_BLOCK2 = 256 tuples, :317-318).
 * hist must hold P counters; key-0 tuples are skipped (:190-192). */
static inline uint32_t glb_dest(uint32_t key, int64_t j, int type, int P, int rank_sets, int ranks_per_set)
{
    uint32_t h = orc_glb_partition_hash(key);
    if (type == 0) return h & (uint32_t)(P - 1);
    uint32_t i = (uint32_t)(j & 255);
    return (h & (uint32_t)(P / rank_sets - 1)) + (i & (uint32_t)(rank_sets - 1)) * (uint32_t)(ranks_per_set * 64);
}

void orc_glb_partition_count(const orc_tuple *t, int64_t n, int type, int P, int rank_sets,
                             int ranks_per_set, uint32_t *hist)
{
    memset(hist, 0, (size_t)P * sizeof(uint32_t));
    for (int64_t j = 0; j < n; j++)
        if (t[j].key) hist[glb_dest(t[j].key, j, type, P, rank_sets, ranks_per_set)]++;
}

/* The destination the count above gives each tuple of one DPU's block (-1 for
 * padding): the partition the packet scatter writes it to
 * (glb_partition_packet.c:430-431, 543-544). */
void orc_glb_partition_dest(const orc_tuple *t, int64_t n, int type, int P, int rank_sets, int ranks_per_set,
                            int32_t *dest)
{
    for (int64_t j = 0; j < n; j++)
        dest[j] = t[j].key ? (int32_t)glb_dest(t[j].key, j, type, P, rank_sets, ranks_per_set) : -1;
}

/* ---------------------------------------------------------- simple join -- */

/* Independent oracle: one open-addressing map over all of R (first R tuple in
 * R order wins for a repeated key), then one pass over S in S order. */
int64_t orc_simple_join(const orc_tuple *R, int64_t nR, const orc_tuple *S, int64_t nS,
                        int keep_unmatched, orc_tuple *out)
{
    int64_t cap = 16;
    while (cap < 2 * nR + 16) cap <<= 1;
    orc_tuple *tab = (orc_tuple *)calloc((size_t)cap, sizeof(orc_tuple));
    if (!tab) return ORC_E_NOMEM;
    uint64_t mask = (uint64_t)cap - 1;
    for (int64_t i = 0; i < nR; i++) {
        uint32_t k = R[i].key;
        if (k == 0) continue;
        uint64_t s = mix64(k) & mask;
        while (tab[s].key != 0 && tab[s].key != k) s = (s + 1) & mask;
        if (tab[s].key == 0) tab[s] = R[i];
    }
    int64_t m = 0;
    for (int64_t i = 0; i < nS; i++) {
        uint32_t k = S[i].key;
        if (k == 0) continue;
        uint64_t s = mix64(k) & mask;
        while (tab[s].key != 0 && tab[s].key != k) s = (s + 1) & mask;
        if (tab[s].key == k) {
            out[m].key = tab[s].pay;
            out[m].pay = S[i].pay;
            m++;
        } else if (keep_unmatched) {
            out[m++] = S[i];
        }
    }
    free(tab);
    return m;
}

/* ------------------------------------------------- reference pipeline ---- */

typedef struct {
    int D;                 /* DPUs = 64 * ranks */
    int ranks, G, rps, B;  /* ranks, rank sets, ranks per set, bank set */
    int alg;
    int64_t per_dpu_R, per_dpu_S;
    const orc_tuple *R, *S;
    int64_t nR, nS;
    /* per (source block, destination) counts, then offsets */
    int64_t *cR, *cS;      /* [D][D] */
    orc_tuple *pR, *pS;    /* partitioned, destination-major */
    int64_t *offR, *offS;  /* [D+1] destination starts */
    /* per-destination outputs */
    orc_tuple **dst_out;
    int64_t *dst_n;
    int err;
} refpipe_t;

static inline int ilog2i(int64_t v) { int l = 0; while ((1ll << l) < v) l++; return l; }

/* LoadColumn's split (query.cc:230-300): pad to a multiple of D*8 bytes (a full
 * extra block when already aligned) and cut into D equal blocks; padding is key 0. */
static int64_t per_dpu_tuples(int64_t n, int D)
{
    int64_t bytes = n * 8, align = (int64_t)D * 8;
    int64_t total = bytes + (align - bytes % align);
    return total / 8 / D;
}

static inline orc_tuple src_tuple(const orc_tuple *base, int64_t n, int64_t per, int blk, int64_t j)
{
    int64_t g = (int64_t)blk * per + j;
    if (g < n) return base[g];
    orc_tuple z = {0, 0};
    return z;
}

/* LUT_BG of glb_chipwise_partition_count.c:132-139, written as a formula:
 * bank-group member k of B sits at chip (k / (B/8)) and bank (k % (B/8)). */
static inline int lut_bg(int B, int k) { int w = B / 8; return (k / w) * 8 + (k % w); }

/* Destination base of bank-group partition `temp` (glb_chipwise_partition_count.c:251-253). */
static inline int bg_base(int B, uint32_t temp)
{
    int per_rank = 64 / B;
    int lg_pr = ilog2i(per_rank), lgB = ilog2i(B);
    return (int)(((temp & (uint32_t)(per_rank - 1)) << (lgB - 3)) + ((temp >> lg_pr) << 6));
}

/* Calls emit(dest) for every DPU that receives R tuple `t` (replicas included). */
#define FOR_R_DESTS(rp, t, DEST_STMT)                                                     \
    do {                                                                                 \
        uint32_t h_ = orc_glb_partition_hash((t).key);                                   \
        if ((rp)->B == 1) {                                                              \
            int PR_ = 64 * (rp)->rps;                                                    \
            int p_ = (int)(h_ & (uint32_t)(PR_ - 1));                                    \
            for (int g_ = 0; g_ < (rp)->G; g_++) { int dest = g_ * PR_ + p_; DEST_STMT; } \
        } else {                                                                         \
            int nBG_ = (rp)->rps * 64 / (rp)->B;                                         \
            uint32_t temp_ = h_ & (uint32_t)(nBG_ - 1);                                  \
            int base_ = bg_base((rp)->B, temp_);                                         \
            int lgset_ = ilog2i(64 * (rp)->rps);                                         \
            for (int g_ = 0; g_ < (rp)->G; g_++)                                         \
                for (int k_ = 0; k_ < (rp)->B; k_++) {                                   \
                    int dest = base_ + lut_bg((rp)->B, k_) + (g_ << lgset_);             \
                    DEST_STMT;                                                           \
                }                                                                        \
        }                                                                                \
    } while (0)

/* Destination of S tuple `t` at index j of its source block. */
static inline int s_dest(const refpipe_t *rp, orc_tuple t, int64_t j)
{
    uint32_t h = orc_glb_partition_hash(t.key);
    int i = (int)(j & 255);
    if (rp->B == 1) {
        int PR = 64 * rp->rps; /* glb_partition_count.c:312-318 */
        return (int)(h & (uint32_t)(PR - 1)) + (i & (rp->G - 1)) * PR;
    }
    int nBG = rp->rps * 64 / rp->B;  /* glb_chipwise_partition_count.c:158-255 */
    uint32_t temp = h & (uint32_t)(nBG - 1);
    int slot = 256 / rp->G;
    return bg_base(rp->B, temp) + lut_bg(rp->B, i & (rp->B - 1)) +
           (((i / slot) & (rp->G - 1)) << ilog2i(64 * rp->rps));
}

/* The chip-wise count kernel's histogram for one DPU's S block (the source
 * block's D = 64 * ranks destinations; glb_chipwise_partition_count.c:158-255):
 * s_dest of every non-padding tuple. bank_set is 8 ... 64 (the kernel only
 * runs with bank sets). Returns 0 or ORC_E_ARG. */
static int chipwise_setup(refpipe_t *rp, int ranks, int rank_sets, int bank_set)
{
    if (ranks <= 0 || rank_sets <= 0 || ranks % rank_sets || rank_sets > 256) return ORC_E_ARG;
    if (!(bank_set == 8 || bank_set == 16 || bank_set == 32 || bank_set == 64)) return ORC_E_ARG;
    memset(rp, 0, sizeof(*rp));
    rp->ranks = ranks; rp->G = rank_sets; rp->rps = ranks / rank_sets; rp->B = bank_set;
    return rp->rps * 64 < bank_set ? ORC_E_ARG : ORC_OK;
}

int orc_chipwise_partition_count(const orc_tuple *t, int64_t n, int ranks, int rank_sets, int bank_set,
                                 uint32_t *hist)
{
    refpipe_t rp;
    const int e = chipwise_setup(&rp, ranks, rank_sets, bank_set);
    if (e) return e;
    memset(hist, 0, (size_t)ranks * 64 * sizeof(uint32_t));
    for (int64_t j = 0; j < n; j++)
        if (t[j].key) hist[s_dest(&rp, t[j], j)]++;
    return ORC_OK;
}

/* The DPUs that receive an R tuple of `key` (replicas included; at most
 * 64 * ranks): FOR_R_DESTS. Returns their number or ORC_E_ARG. */
int orc_r_dests(uint32_t key, int ranks, int rank_sets, int bank_set, int32_t *dests)
{
    refpipe_t rp;
    int e = bank_set == 1 ? ORC_OK : chipwise_setup(&rp, ranks, rank_sets, bank_set);
    if (e) return e;
    if (bank_set == 1) {
        if (ranks <= 0 || rank_sets <= 0 || ranks % rank_sets) return ORC_E_ARG;
        memset(&rp, 0, sizeof(rp));
        rp.ranks = ranks; rp.G = rank_sets; rp.rps = ranks / rank_sets; rp.B = 1;
    }
    orc_tuple t = {key, 0};
    int m = 0;
    FOR_R_DESTS(&rp, t, dests[m++] = dest);
    return m;
}

/* Each tuple's destination under the chip-wise split (-1 for padding): where
 * glb_chipwise_partition_packet.c:468-472 scatters it. */
int orc_chipwise_partition_dest(const orc_tuple *t, int64_t n, int ranks, int rank_sets, int bank_set,
                                int32_t *dest)
{
    refpipe_t rp;
    const int e = chipwise_setup(&rp, ranks, rank_sets, bank_set);
    if (e) return e;
    for (int64_t j = 0; j < n; j++) dest[j] = t[j].key ? s_dest(&rp, t[j], j) : -1;
    return ORC_OK;
}

static void count_task(void *ctx, int64_t blk)
{
    refpipe_t *rp = (refpipe_t *)ctx;
    int64_t *cr = rp->cR + blk * rp->D, *cs = rp->cS + blk * rp->D;
    for (int64_t j = 0; j < rp->per_dpu_R; j++) {
        orc_tuple t = src_tuple(rp->R, rp->nR, rp->per_dpu_R, (int)blk, j);
        if (t.key == 0) continue;
        FOR_R_DESTS(rp, t, cr[dest]++);
    }
    for (int64_t j = 0; j < rp->per_dpu_S; j++) {
        orc_tuple t = src_tuple(rp->S, rp->nS, rp->per_dpu_S, (int)blk, j);
        if (t.key == 0) continue;
        cs[s_dest(rp, t, j)]++;
    }
}

static void scatter_task(void *ctx, int64_t blk)
{
    refpipe_t *rp = (refpipe_t *)ctx;
    int64_t *cr = rp->cR + blk * rp->D, *cs = rp->cS + blk * rp->D;
    for (int64_t j = 0; j < rp->per_dpu_R; j++) {
        orc_tuple t = src_tuple(rp->R, rp->nR, rp->per_dpu_R, (int)blk, j);
        if (t.key == 0) continue;
        FOR_R_DESTS(rp, t, rp->pR[cr[dest]++] = t);
    }
    for (int64_t j = 0; j < rp->per_dpu_S; j++) {
        orc_tuple t = src_tuple(rp->S, rp->nS, rp->per_dpu_S, (int)blk, j);
        if (t.key == 0) continue;
        rp->pS[cs[s_dest(rp, t, j)]++] = t;
    }
}

/* Per-DPU hash join: local partitioning, 4096-slot linear-probe build, probe. */
static int dpu_phj(const orc_tuple *r, int64_t nr, const orc_tuple *s, int64_t ns, orc_tuple *out,
                   int64_t *nout)
{
    /* a2a_packetwise_srj_local_partition.c:323-341: L = 2^bitlen(nr / 1935). */
    int64_t temp = nr / 1935;
    int64_t L = 1;
    while (temp > 0) { temp >>= 1; L <<= 1; }
    int64_t *rc = (int64_t *)calloc((size_t)L + 1, sizeof(int64_t));
    int64_t *sc = (int64_t *)calloc((size_t)L + 1, sizeof(int64_t));
    orc_tuple *rl = (orc_tuple *)malloc((size_t)(nr ? nr : 1) * sizeof(orc_tuple));
    orc_tuple *sl = (orc_tuple *)malloc((size_t)(ns ? ns : 1) * sizeof(orc_tuple));
    orc_tuple *tab = (orc_tuple *)malloc(4096 * sizeof(orc_tuple));
    if (!rc || !sc || !rl || !sl || !tab) {
        free(rc); free(sc); free(rl); free(sl); free(tab);
        return ORC_E_NOMEM;
    }
    uint32_t mask = (uint32_t)(L - 1);
    for (int64_t i = 0; i < nr; i++) rc[(orc_local_partition_hash(r[i].key) & mask) + 1]++;
    for (int64_t i = 0; i < ns; i++) sc[(orc_local_partition_hash(s[i].key) & mask) + 1]++;
    for (int64_t l = 0; l < L; l++) { rc[l + 1] += rc[l]; sc[l + 1] += sc[l]; }
    {
        int64_t *cur = (int64_t *)malloc((size_t)L * sizeof(int64_t));
        if (!cur) { free(rc); free(sc); free(rl); free(sl); free(tab); return ORC_E_NOMEM; }
        memcpy(cur, rc, (size_t)L * sizeof(int64_t));
        for (int64_t i = 0; i < nr; i++) rl[cur[orc_local_partition_hash(r[i].key) & mask]++] = r[i];
        memcpy(cur, sc, (size_t)L * sizeof(int64_t));
        for (int64_t i = 0; i < ns; i++) sl[cur[orc_local_partition_hash(s[i].key) & mask]++] = s[i];
        free(cur);
    }
    int rc_err = ORC_OK;
    int64_t m = 0;
    for (int64_t l = 0; l < L && rc_err == ORC_OK; l++) {
        int64_t r0 = rc[l], r1 = rc[l + 1];
        if (r1 - r0 > 4096) { rc_err = ORC_E_TABLE_FULL; break; }
        memset(tab, 0, 4096 * sizeof(orc_tuple));
        /* a2a_srj_build.c:202-295: slot = join_hash & 0xFFF, linear probing with wrap. */
        for (int64_t i = r0; i < r1; i++) {
            uint32_t slot = orc_join_hash(rl[i].key) & 0xFFFu;
            while (tab[slot].key != 0) slot = (slot + 1) & 0xFFFu;
            tab[slot] = rl[i];
        }
        /* a2a_srj_probe_inner_mt.c:101-168: stop at empty (miss) or equal key (hit,
         * emit and stop: first match only); give up after 4097 steps. */
        for (int64_t i = sc[l]; i < sc[l + 1]; i++) {
            uint32_t key = sl[i].key, slot = orc_join_hash(key) & 0xFFFu;
            for (int runs = 0; runs <= 4096; runs++) {
                if (tab[slot].key == 0) break;
                if (tab[slot].key == key) {
                    out[m].key = tab[slot].pay;
                    out[m].pay = sl[i].pay;
                    m++;
                    break;
                }
                slot = (slot + 1) & 0xFFFu;
            }
        }
    }
    free(rc); free(sc); free(rl); free(sl); free(tab);
    *nout = m;
    return rc_err;
}

/* The local partition count of dpu_phj for nr R tuples. */
int64_t orc_local_partitions(int64_t nr)
{
    int64_t temp = nr / 1935, L = 1;
    while (temp > 0) { temp >>= 1; L <<= 1; }
    return L;
}

/* The layout dpu_phj joins: t grouped by local_partition_hash & (L-1), input
 * order kept within a group; off[0..L] receives the group starts (L a power of
 * two). Exported for the checks against the reference's own build and probe
 * kernels, which take their input in this layout. */
int orc_local_partition(const orc_tuple *t, int64_t n, int64_t L, orc_tuple *out, int64_t *off)
{
    if (L < 1 || (L & (L - 1)) || n < 0) return ORC_E_ARG;
    const uint32_t mask = (uint32_t)(L - 1);
    memset(off, 0, (size_t)(L + 1) * sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) off[(orc_local_partition_hash(t[i].key) & mask) + 1]++;
    for (int64_t l = 0; l < L; l++) off[l + 1] += off[l];
    int64_t *cur = (int64_t *)malloc((size_t)L * sizeof(int64_t));
    if (!cur) return ORC_E_NOMEM;
    memcpy(cur, off, (size_t)L * sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) out[cur[orc_local_partition_hash(t[i].key) & mask]++] = t[i];
    free(cur);
    return ORC_OK;
}

/* One DPU's hash join as dpu_phj restates it: the pairs written to out (room
 * for ns) or an ORC_E_ code. */
int64_t orc_dpu_phj(const orc_tuple *r, int64_t nr, const orc_tuple *s, int64_t ns, orc_tuple *out)
{
    int64_t m = 0;
    const int rc = dpu_phj(r, nr, s, ns, out, &m);
    return rc ? rc : m;
}

static int cmp_key_stable(const void *a, const void *b)
{
    const orc_tuple *x = (const orc_tuple *)a, *y = (const orc_tuple *)b;
    return (x->key > y->key) - (x->key < y->key);
}

/* Per-DPU sort-merge (mpsm_join_sort_probe.c:152-236): both sides sorted by key,
 * merge; each S tuple takes the first R tuple with its key, else stays unchanged.
 * The reference stops probing a bucket at the first S key below the current R
 * key (:226-229), which leaves later S tuples unmatched only when S holds keys
 * that R lacks; this restatement keeps merging (intended semantics). It also
 * joins every S tuple, where the reference's sort-probe leaves bucket 511 of
 * each block of 512 range buckets and the last bucket unprobed (:297, :395) and
 * reads a stale buffer for a bucket of one tuple (its merge sort, :153-208). On
 * the buckets it does join, the two agree (the reference's kernels run on the
 * host in the tests). */
static int dpu_smj(const orc_tuple *r, int64_t nr, const orc_tuple *s, int64_t ns, orc_tuple *out,
                   int64_t *nout)
{
    /* R sorted by (key, position): among equal keys the first R tuple comes first,
     * as the stable merge sort of the reference leaves them. */
    orc_tuple *kx = (orc_tuple *)malloc((size_t)(nr ? nr : 1) * sizeof(orc_tuple));
    orc_tuple *rs = (orc_tuple *)malloc((size_t)(nr ? nr : 1) * sizeof(orc_tuple));
    if (!kx || !rs) { free(kx); free(rs); return ORC_E_NOMEM; }
    for (int64_t i = 0; i < nr; i++) { kx[i].key = r[i].key; kx[i].pay = (uint32_t)i; }
    if (orc_sort_pairs(kx, nr) != ORC_OK) { free(kx); free(rs); return ORC_E_NOMEM; }
    for (int64_t i = 0; i < nr; i++) rs[i] = r[kx[i].pay];
    free(kx);
    memcpy(out, s, (size_t)ns * sizeof(orc_tuple));
    qsort(out, (size_t)ns, sizeof(orc_tuple), cmp_key_stable);
    int64_t ri = 0;
    for (int64_t i = 0; i < ns; i++) {
        uint32_t k = out[i].key;
        while (ri < nr && rs[ri].key < k) ri++;
        if (ri < nr && rs[ri].key == k) out[i].key = rs[ri].pay;
    }
    free(rs);
    *nout = ns;
    return ORC_OK;
}

/* One DPU's sort-merge join as dpu_smj restates it: all n_s S tuples, sorted by
 * key, matched ones carrying their R payload as key. Returns n_s or an error. */
int64_t orc_dpu_smj(const orc_tuple *r, int64_t nr, const orc_tuple *s, int64_t ns, orc_tuple *out)
{
    int64_t m = 0;
    const int rc = dpu_smj(r, nr, s, ns, out, &m);
    return rc ? rc : m;
}

/* Per-DPU nested loop (nested_loop_join.c:184-231): every S tuple is compared
 * with the R tuples in R order and takes the first equal key; unmatched S tuples
 * stay unchanged. Restated with a first-occurrence map, which yields the same
 * rows. (The reference keeps comparing the rewritten value against later R
 * blocks, :156-231, so a payload that equals a later R key is rewritten again;
 * this restatement keeps the single rewrite the kernel intends. It also compares
 * key 0, so its (0, 0) padding "joins" R's padding and stays (0, 0); padding
 * gives no row here.) */
static int dpu_nl(const orc_tuple *r, int64_t nr, const orc_tuple *s, int64_t ns, orc_tuple *out,
                  int64_t *nout)
{
    int64_t m = orc_simple_join(r, nr, s, ns, 1, out);
    if (m < 0) return (int)m;
    *nout = m;
    return ORC_OK;
}

static void local_task(void *ctx, int64_t d)
{
    refpipe_t *rp = (refpipe_t *)ctx;
    const orc_tuple *r = rp->pR + rp->offR[d], *s = rp->pS + rp->offS[d];
    int64_t nr = rp->offR[d + 1] - rp->offR[d], ns = rp->offS[d + 1] - rp->offS[d];
    orc_tuple *out = (orc_tuple *)malloc((size_t)(ns ? ns : 1) * sizeof(orc_tuple));
    if (!out) { rp->err = ORC_E_NOMEM; return; }
    int64_t m = 0;
    int e;
    if (rp->alg == ORC_ALG_SMJ) e = dpu_smj(r, nr, s, ns, out, &m);
    else if (rp->alg == ORC_ALG_NL) e = dpu_nl(r, nr, s, ns, out, &m);
    else e = dpu_phj(r, nr, s, ns, out, &m);
    if (e != ORC_OK) rp->err = e;
    rp->dst_out[d] = out;
    rp->dst_n[d] = m;
}

static void free_refpipe(refpipe_t *rp)
{
    if (rp->dst_out)
        for (int d = 0; d < rp->D; d++) free(rp->dst_out[d]);
    free(rp->dst_out); free(rp->dst_n);
    free(rp->cR); free(rp->cS); free(rp->pR); free(rp->pS); free(rp->offR); free(rp->offS);
}

static int is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

static int refpipe_setup(refpipe_t *rp, const orc_tuple *R, int64_t nR, const orc_tuple *S, int64_t nS,
                         int ranks, int rank_sets, int bank_set, int alg)
{
    memset(rp, 0, sizeof(*rp));
    if (nR < 0 || nS < 0 || ranks <= 0 || rank_sets <= 0 || ranks % rank_sets) return ORC_E_ARG;
    if (!is_pow2(ranks / rank_sets) || !is_pow2(rank_sets) || rank_sets > 256) return ORC_E_ARG;
    /* pipeline.cc:256-260 accepts bank_set in {1, 8, 16, 32, 64} */
    if (!(bank_set == 1 || bank_set == 8 || bank_set == 16 || bank_set == 32 || bank_set == 64))
        return ORC_E_ARG;
    if (alg < 0 || alg > 3) return ORC_E_ARG;
    rp->ranks = ranks; rp->G = rank_sets; rp->rps = ranks / rank_sets; rp->B = bank_set;
    rp->D = 64 * ranks; rp->alg = alg;
    rp->R = R; rp->S = S; rp->nR = nR; rp->nS = nS;
    rp->per_dpu_R = per_dpu_tuples(nR, rp->D);
    rp->per_dpu_S = per_dpu_tuples(nS, rp->D);
    return ORC_OK;
}

static int refpipe_partition(refpipe_t *rp, int nthreads)
{
    int D = rp->D;
    rp->cR = (int64_t *)calloc((size_t)D * D, sizeof(int64_t));
    rp->cS = (int64_t *)calloc((size_t)D * D, sizeof(int64_t));
    rp->offR = (int64_t *)calloc((size_t)D + 1, sizeof(int64_t));
    rp->offS = (int64_t *)calloc((size_t)D + 1, sizeof(int64_t));
    if (!rp->cR || !rp->cS || !rp->offR || !rp->offS) return ORC_E_NOMEM;
    parallel_for(nthreads, D, count_task, rp);
    /* destination-major offsets: dest d, then source block order */
    int64_t runR = 0, runS = 0;
    for (int d = 0; d < D; d++) {
        rp->offR[d] = runR; rp->offS[d] = runS;
        for (int b = 0; b < D; b++) {
            int64_t c = rp->cR[(int64_t)b * D + d]; rp->cR[(int64_t)b * D + d] = runR; runR += c;
            c = rp->cS[(int64_t)b * D + d]; rp->cS[(int64_t)b * D + d] = runS; runS += c;
        }
    }
    rp->offR[D] = runR; rp->offS[D] = runS;
    rp->pR = (orc_tuple *)malloc((size_t)(runR ? runR : 1) * sizeof(orc_tuple));
    rp->pS = (orc_tuple *)malloc((size_t)(runS ? runS : 1) * sizeof(orc_tuple));
    if (!rp->pR || !rp->pS) return ORC_E_NOMEM;
    parallel_for(nthreads, D, scatter_task, rp);
    return ORC_OK;
}

/* Per-DPU R and S tuple counts after global partitioning and replication
 * (what each DPU holds when the local join starts). */
int orc_refpipe_dpu_sizes(const orc_tuple *R, int64_t nR, const orc_tuple *S, int64_t nS, int ranks,
                          int rank_sets, int bank_set, int nthreads, int64_t *r_sizes, int64_t *s_sizes)
{
    refpipe_t rp;
    int e = refpipe_setup(&rp, R, nR, S, nS, ranks, rank_sets, bank_set, 0);
    if (e) return e;
    e = refpipe_partition(&rp, nthreads);
    if (e == ORC_OK)
        for (int d = 0; d < rp.D; d++) {
            r_sizes[d] = rp.offR[d + 1] - rp.offR[d];
            s_sizes[d] = rp.offS[d + 1] - rp.offS[d];
        }
    free_refpipe(&rp);
    return e;
}

/* Whole reference pipeline: split, global partition + replication, per-DPU local
 * join, concatenation of the DPU outputs in DPU order (src/queryHostFunc.cc:1058-1126
 * returns them per rank; padding is not emitted). Returns the pair count or a
 * negative ORC_E_* code. `out` must hold nS pairs. */
int64_t orc_refpipe_join(const orc_tuple *R, int64_t nR, const orc_tuple *S, int64_t nS, int ranks,
                         int rank_sets, int bank_set, int alg, int nthreads, orc_tuple *out)
{
    refpipe_t rp;
    int e = refpipe_setup(&rp, R, nR, S, nS, ranks, rank_sets, bank_set, alg == ORC_ALG_NPHJ ? 0 : alg);
    if (e) return e;
    e = refpipe_partition(&rp, nthreads);
    if (e) { free_refpipe(&rp); return e; }
    rp.dst_out = (orc_tuple **)calloc((size_t)rp.D, sizeof(orc_tuple *));
    rp.dst_n = (int64_t *)calloc((size_t)rp.D, sizeof(int64_t));
    if (!rp.dst_out || !rp.dst_n) { free_refpipe(&rp); return ORC_E_NOMEM; }
    parallel_for(nthreads, rp.D, local_task, &rp);
    if (rp.err) { int err = rp.err; free_refpipe(&rp); return err; }
    int64_t m = 0;
    for (int d = 0; d < rp.D; d++) {
        memcpy(out + m, rp.dst_out[d], (size_t)rp.dst_n[d] * sizeof(orc_tuple));
        m += rp.dst_n[d];
    }
    free_refpipe(&rp);
    return m;
}

/* ------------------------------------------- threaded checker utilities -- */

/* orc_simple_join with threads, for full-size checks (2^27 R x 2^29 S): the
 * table maps a key to the smallest R index holding it (a CAS keeps the minimum),
 * which is exactly the single-threaded rule "first R tuple in R order wins";
 * S is probed in contiguous slices whose outputs are concatenated in S order.
 * The result is byte-identical to orc_simple_join. */
typedef struct {
    const orc_tuple *R, *S;
    int64_t nR, nS;
    uint64_t *tab;   /* (key << 32 | R index + 1), 0 = empty */
    uint64_t mask;
    int keep;
    int64_t slices, per;
    int64_t *cnt;    /* matches per S slice, then the slice's output offset */
    orc_tuple *out;
    int pass;        /* 0 build, 1 count, 2 write */
} sj_mt_t;

static void sj_build_task(void *ctx, int64_t t)
{
    sj_mt_t *c = (sj_mt_t *)ctx;
    int64_t b = c->per * t, e = b + c->per < c->nR ? b + c->per : c->nR;
    for (int64_t i = b; i < e; i++) {
        uint32_t k = c->R[i].key;
        if (k == 0) continue;
        uint64_t ent = ((uint64_t)k << 32) | (uint64_t)(i + 1);
        uint64_t s = mix64(k) & c->mask;
        for (;;) {
            uint64_t cur = __atomic_load_n(&c->tab[s], __ATOMIC_RELAXED);
            if (cur == 0) {
                if (__atomic_compare_exchange_n(&c->tab[s], &cur, ent, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                    break;
                continue;  /* cur now holds the winner: look at it again */
            }
            if ((uint32_t)(cur >> 32) == k) {
                if ((uint32_t)cur <= (uint32_t)(i + 1)) break;
                if (__atomic_compare_exchange_n(&c->tab[s], &cur, ent, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                    break;
                continue;
            }
            s = (s + 1) & c->mask;
        }
    }
}

static void sj_probe_task(void *ctx, int64_t t)
{
    sj_mt_t *c = (sj_mt_t *)ctx;
    int64_t b = c->per * t, e = b + c->per < c->nS ? b + c->per : c->nS;
    int64_t m = c->pass == 2 ? c->cnt[t] : 0;
    for (int64_t i = b; i < e; i++) {
        uint32_t k = c->S[i].key;
        if (k == 0) continue;
        uint64_t s = mix64(k) & c->mask, ent;
        while ((ent = c->tab[s]) != 0 && (uint32_t)(ent >> 32) != k) s = (s + 1) & c->mask;
        if (ent) {
            if (c->pass == 2) {
                c->out[m].key = c->R[(uint32_t)ent - 1].pay;
                c->out[m].pay = c->S[i].pay;
            }
            m++;
        } else if (c->keep) {
            if (c->pass == 2) c->out[m] = c->S[i];
            m++;
        }
    }
    if (c->pass == 1) c->cnt[t] = m;
}

int64_t orc_simple_join_mt(const orc_tuple *R, int64_t nR, const orc_tuple *S, int64_t nS, int keep_unmatched,
                           int nthreads, orc_tuple *out)
{
    if (nR < 0 || nS < 0 || nR >= 0xFFFFFFFFll) return ORC_E_ARG;
    if (nthreads < 1) nthreads = 1;
    sj_mt_t c;
    memset(&c, 0, sizeof(c));
    c.R = R; c.S = S; c.nR = nR; c.nS = nS; c.keep = keep_unmatched; c.out = out;
    int64_t cap = 16;
    while (cap < 2 * nR + 16) cap <<= 1;
    c.mask = (uint64_t)cap - 1;
    c.tab = (uint64_t *)calloc((size_t)cap, sizeof(uint64_t));
    int64_t slices = 4 * (int64_t)nthreads;
    c.cnt = (int64_t *)calloc((size_t)slices, sizeof(int64_t));
    if (!c.tab || !c.cnt) { free(c.tab); free(c.cnt); return ORC_E_NOMEM; }
    c.per = (nR + slices - 1) / slices;
    if (c.per < 1) c.per = 1;
    parallel_for(nthreads, slices, sj_build_task, &c);
    c.per = (nS + slices - 1) / slices;
    if (c.per < 1) c.per = 1;
    c.pass = 1;
    parallel_for(nthreads, slices, sj_probe_task, &c);
    int64_t run = 0;
    for (int64_t t = 0; t < slices; t++) { int64_t v = c.cnt[t]; c.cnt[t] = run; run += v; }
    c.pass = 2;
    parallel_for(nthreads, slices, sj_probe_task, &c);
    free(c.tab);
    free(c.cnt);
    return run;
}

/* orc_sort_pairs with threads: LSD radix sort, 4 x 16-bit digits, each pass a
 * per-slice count, one exclusive scan in (digit, slice) order and a per-slice
 * scatter, so every pass is stable and the result equals orc_sort_pairs. */
typedef struct {
    uint64_t *a, *b;
    int64_t n, per, slices;
    int64_t *cnt;  /* [slices][65536] */
    int sh;
    int phase;     /* 0 count, 1 scatter */
} rs_mt_t;

static void rs_task(void *ctx, int64_t t)
{
    rs_mt_t *c = (rs_mt_t *)ctx;
    int64_t b = c->per * t, e = b + c->per < c->n ? b + c->per : c->n;
    int64_t *h = c->cnt + (size_t)t * 65536;
    if (c->phase == 0) {
        memset(h, 0, 65536 * sizeof(int64_t));
        for (int64_t i = b; i < e; i++) h[(c->a[i] >> c->sh) & 0xffff]++;
    } else {
        for (int64_t i = b; i < e; i++) c->b[h[(c->a[i] >> c->sh) & 0xffff]++] = c->a[i];
    }
}

typedef struct { orc_tuple *p; uint64_t *a; int64_t n, per; int dir; } pack_t;

static void pack_task(void *ctx, int64_t t)
{
    pack_t *c = (pack_t *)ctx;
    int64_t b = c->per * t, e = b + c->per < c->n ? b + c->per : c->n;
    if (c->dir == 0)
        for (int64_t i = b; i < e; i++) c->a[i] = ((uint64_t)c->p[i].key << 32) | c->p[i].pay;
    else
        for (int64_t i = b; i < e; i++) { c->p[i].key = (uint32_t)(c->a[i] >> 32); c->p[i].pay = (uint32_t)c->a[i]; }
}

int orc_sort_pairs_mt(orc_tuple *p, int64_t n, int nthreads)
{
    if (n <= 1) return ORC_OK;
    if (nthreads < 1) nthreads = 1;
    rs_mt_t c;
    memset(&c, 0, sizeof(c));
    c.n = n;
    c.slices = nthreads;
    c.per = (n + c.slices - 1) / c.slices;
    c.a = (uint64_t *)malloc((size_t)n * 8);
    c.b = (uint64_t *)malloc((size_t)n * 8);
    c.cnt = (int64_t *)malloc((size_t)c.slices * 65536 * sizeof(int64_t));
    if (!c.a || !c.b || !c.cnt) { free(c.a); free(c.b); free(c.cnt); return ORC_E_NOMEM; }
    pack_t pk = {p, c.a, n, c.per, 0};
    parallel_for(nthreads, c.slices, pack_task, &pk);
    for (int pass = 0; pass < 4; pass++) {
        c.sh = 16 * pass;
        c.phase = 0;
        parallel_for(nthreads, c.slices, rs_task, &c);
        int64_t run = 0;
        for (int d = 0; d < 65536; d++)
            for (int64_t t = 0; t < c.slices; t++) {
                int64_t v = c.cnt[(size_t)t * 65536 + d];
                c.cnt[(size_t)t * 65536 + d] = run;
                run += v;
            }
        c.phase = 1;
        parallel_for(nthreads, c.slices, rs_task, &c);
        uint64_t *tmp = c.a; c.a = c.b; c.b = tmp;
    }
    pk.a = c.a;
    pk.dir = 1;
    parallel_for(nthreads, c.slices, pack_task, &pk);
    free(c.a); free(c.b); free(c.cnt);
    return ORC_OK;
}

/* --------------------------------------------- benchmark-relation generator -- */

/* The seeded relations of the benchmark, restated for the checker and for the
 * CPU arms of the benchmark so that they need no product library: the same
 * definitions as the product's generator, value for value (a CPU test compares
 * the two on the host, a GPU test this one with the device's R and uniform S).
 *   R[i] = (1 + perm_R(i), i): keys a permutation of 1..nR, payload the row id;
 *   S[j] = (R[m(j)].key, j), m(j) uniform (zipf 0) or perm_rank(zipf_rank(j) - 1).
 * Pieces: splitmix64 (Steele, Lea, Flood 2014); a 4-round unbalanced Feistel
 * network on ceil(log2 n) bits with cycle-walking as the permutation; Zipf ranks
 * by rejection-inversion (Hoermann and Derflinger, ACM TOMACS 6(3), 1996). */
typedef struct { uint64_t n, seed; int lo_bits, hi_bits; } g_perm;

static g_perm g_make_perm(uint64_t n, uint64_t seed)
{
    g_perm p;
    p.n = n;
    p.seed = seed;
    int b = 2;
    while ((1ull << b) < n) b++;
    p.lo_bits = b / 2;
    p.hi_bits = b - p.lo_bits;
    return p;
}

static uint64_t g_feistel(const g_perm *p, uint64_t x)
{
    const uint64_t lo_mask = (1ull << p->lo_bits) - 1, hi_mask = (1ull << p->hi_bits) - 1;
    uint64_t lo = x & lo_mask, hi = x >> p->lo_bits;
    for (int r = 0; r < 4; r += 2) {
        hi ^= mix64(p->seed + 0x9e3779b97f4a7c15ull * (uint64_t)(r + 1) + lo) & hi_mask;
        lo ^= mix64(p->seed + 0x9e3779b97f4a7c15ull * (uint64_t)(r + 2) + hi) & lo_mask;
    }
    return (hi << p->lo_bits) | lo;
}

static uint64_t g_perm_apply(const g_perm *p, uint64_t x)
{
    uint64_t y = g_feistel(p, x);
    while (y >= p->n) y = g_feistel(p, y);
    return y;
}

static double g_unit(uint64_t seed, uint64_t idx, uint32_t attempt)
{
    uint64_t z = mix64(seed ^ mix64(idx * 0x9e3779b97f4a7c15ull + attempt));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

typedef struct { double s, h_lo, h_hi, squeeze; uint64_t n; } g_zipf;

static double g_rlog1p(double x) { return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x)); }
static double g_rexpm1(double x) { return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + 0.5 * x * (1.0 + (x / 3.0) * (1.0 + 0.25 * x)); }
static double g_H(const g_zipf *z, double x) { double lx = log(x); return g_rexpm1((1.0 - z->s) * lx) * lx; }
static double g_Hinv(const g_zipf *z, double y)
{
    double t = y * (1.0 - z->s);
    if (t < -1.0) t = -1.0;
    return exp(g_rlog1p(t) * y);
}
static double g_h(const g_zipf *z, double x) { return exp(-z->s * log(x)); }

static g_zipf g_make_zipf(uint64_t n, double s)
{
    g_zipf z;
    z.s = s;
    z.n = n;
    z.h_lo = g_H(&z, 1.5) - 1.0;
    z.h_hi = g_H(&z, (double)n + 0.5);
    z.squeeze = 2.0 - g_Hinv(&z, g_H(&z, 2.5) - g_h(&z, 2.0));
    return z;
}

static uint64_t g_zipf_rank(const g_zipf *z, uint64_t seed, uint64_t idx)
{
    for (uint32_t a = 0;; a++) {
        double y = z->h_hi + g_unit(seed, idx, a) * (z->h_lo - z->h_hi);
        double x = g_Hinv(z, y);
        double kd = x + 0.5;
        uint64_t k = kd < 1.0 ? 1 : (uint64_t)kd;
        if (k > z->n) k = z->n;
        if ((double)k - x <= z->squeeze || y >= g_H(z, (double)k + 0.5) - g_h(z, (double)k)) return k;
        if (a > 1000) return k;
    }
}

static uint64_t g_seed_R(uint64_t s) { return mix64(s ^ 0x52454c4154494f4eull); }
static uint64_t g_seed_rank(uint64_t s) { return mix64(s ^ 0x52414e4b4f524452ull); }
static uint64_t g_seed_S(uint64_t s) { return mix64(s ^ 0x535354524541414dull); }

typedef struct {
    uint64_t seed, nR, nS;
    double zipf;
    g_perm pr, prank;
    g_zipf z;
    orc_tuple *R, *S;
    int64_t slices;
    uint64_t *part;  /* per-slice checksum of the expected pairs */
} gen_t;

static void gen_task(void *ctx, int64_t t)
{
    gen_t *g = (gen_t *)ctx;
    if (g->R) {
        uint64_t b = g->nR * (uint64_t)t / (uint64_t)g->slices, e = g->nR * (uint64_t)(t + 1) / (uint64_t)g->slices;
        for (uint64_t i = b; i < e; i++) {
            g->R[i].key = (uint32_t)(1 + g_perm_apply(&g->pr, i));
            g->R[i].pay = (uint32_t)i;
        }
    }
    uint64_t b = g->nS * (uint64_t)t / (uint64_t)g->slices, e = g->nS * (uint64_t)(t + 1) / (uint64_t)g->slices;
    uint64_t acc = 0;
    const uint64_t ss = g_seed_S(g->seed);
    for (uint64_t j = b; j < e; j++) {
        uint64_t row;
        if (g->zipf <= 0.0)
            row = (uint64_t)(((unsigned __int128)mix64(ss ^ (j * 0x9e3779b97f4a7c15ull)) * g->nR) >> 64);
        else
            row = g_perm_apply(&g->prank, g_zipf_rank(&g->z, ss, j) - 1);
        if (g->S) {
            g->S[j].key = (uint32_t)(1 + g_perm_apply(&g->pr, row));
            g->S[j].pay = (uint32_t)j;
        }
        acc += mix64(((uint64_t)(uint32_t)row << 32) | (uint32_t)j);
    }
    g->part[t] = acc;
}

/* Fills R (nR tuples) and S (nS tuples; either may be NULL) and returns in
 * *expect the checksum of the join's expected output {(m(j), j)}. */
int orc_generate(uint64_t seed, int64_t nR, int64_t nS, double zipf_s, orc_tuple *R, orc_tuple *S,
                 uint64_t *expect, int nthreads)
{
    if (nR <= 0 || nS < 0 || nR >= 0xFFFFFFFFll || zipf_s < 0) return ORC_E_ARG;
    if (nthreads < 1) nthreads = 1;
    gen_t g;
    memset(&g, 0, sizeof(g));
    g.seed = seed; g.nR = (uint64_t)nR; g.nS = (uint64_t)nS; g.zipf = zipf_s;
    g.pr = g_make_perm(g.nR, g_seed_R(seed));
    g.prank = g_make_perm(g.nR, g_seed_rank(seed));
    g.z = g_make_zipf(g.nR, zipf_s > 0 ? zipf_s : 1.0);
    g.R = R; g.S = S;
    g.slices = 8 * (int64_t)nthreads;
    g.part = (uint64_t *)calloc((size_t)g.slices, sizeof(uint64_t));
    if (!g.part) return ORC_E_NOMEM;
    parallel_for(nthreads, g.slices, gen_task, &g);
    uint64_t s = 0;
    for (int64_t t = 0; t < g.slices; t++) s += g.part[t];
    free(g.part);
    if (expect) *expect = s;
    return ORC_OK;
}
