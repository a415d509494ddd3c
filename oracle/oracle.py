"""ctypes view of the oracle (oracle/liboracle.so).

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` import this module, as the checker or as the timed CPU
baseline. The product library never depends on it.

Arrays are numpy ``uint32`` arrays of shape (n, 2): column 0 = key (lvalue),
column 1 = payload (rvalue), the layout of the reference's ``kv_pair_t``
(include/type_defs.hpp:53-56 in yonsei-hpcp/spid-join).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HASH_PATH = os.path.join(HERE, "_ref", "libref_hash.so")

ALG_PHJ, ALG_NPHJ, ALG_SMJ, ALG_NL = 0, 1, 2, 3
ERRORS = {-1: "bad argument", -2: "out of memory", -3: "local partition exceeds 4096 tuples"}

_lib = None


def build():
    """Compile liboracle.so (and the reference hash library when the reference tree exists)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all", "ref-if-present"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32, i64, i32 = ctypes.c_uint32, ctypes.c_int64, ctypes.c_int
        vp = ctypes.c_void_p
        for f in ("orc_glb_partition_hash", "orc_local_partition_hash", "orc_join_hash", "orc_join_hash2"):
            getattr(L, f).restype = u32
            getattr(L, f).argtypes = [u32]
        L.orc_crc_table.restype = ctypes.POINTER(u32)
        L.orc_checksum.restype = ctypes.c_uint64
        L.orc_checksum.argtypes = [vp, i64]
        L.orc_sort_pairs.restype = i32
        L.orc_sort_pairs.argtypes = [vp, i64]
        L.orc_glb_partition_count.restype = None
        L.orc_glb_partition_count.argtypes = [vp, i64, i32, i32, i32, i32, vp]
        L.orc_simple_join.restype = i64
        L.orc_simple_join.argtypes = [vp, i64, vp, i64, i32, vp]
        L.orc_refpipe_join.restype = i64
        L.orc_refpipe_join.argtypes = [vp, i64, vp, i64, i32, i32, i32, i32, i32, vp]
        L.orc_simple_join_mt.restype = i64
        L.orc_simple_join_mt.argtypes = [vp, i64, vp, i64, i32, i32, vp]
        L.orc_sort_pairs_mt.restype = i32
        L.orc_sort_pairs_mt.argtypes = [vp, i64, i32]
        L.orc_generate.restype = i32
        L.orc_generate.argtypes = [ctypes.c_uint64, i64, i64, ctypes.c_double, vp, vp,
                                   ctypes.POINTER(ctypes.c_uint64), i32]
        L.orc_local_partitions.restype = i64
        L.orc_local_partitions.argtypes = [i64]
        L.orc_local_partition.restype = i32
        L.orc_local_partition.argtypes = [vp, i64, i64, vp, vp]
        L.orc_dpu_phj.restype = i64
        L.orc_dpu_phj.argtypes = [vp, i64, vp, i64, vp]
        L.orc_glb_partition_dest.restype = None
        L.orc_glb_partition_dest.argtypes = [vp, i64, i32, i32, i32, i32, vp]
        L.orc_r_dests.restype = i32
        L.orc_r_dests.argtypes = [ctypes.c_uint32, i32, i32, i32, vp]
        L.orc_chipwise_partition_dest.restype = i32
        L.orc_chipwise_partition_dest.argtypes = [vp, i64, i32, i32, i32, vp]
        L.orc_chipwise_partition_count.restype = i32
        L.orc_chipwise_partition_count.argtypes = [vp, i64, i32, i32, i32, vp]
        L.orc_dpu_smj.restype = i64
        L.orc_dpu_smj.argtypes = [vp, i64, vp, i64, vp]
        L.orc_refpipe_dpu_sizes.restype = i32
        L.orc_refpipe_dpu_sizes.argtypes = [vp, i64, vp, i64, i32, i32, i32, i32, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _tuples(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if a.ndim != 2 or a.shape[1] != 2:
        raise ValueError("tuples must have shape (n, 2)")
    return a


def hashes(keys):
    """(glb_partition_hash, local_partition_hash, join_hash, join_hash2) per key."""
    L = lib()
    out = np.zeros((len(keys), 4), dtype=np.uint32)
    for i, k in enumerate(keys):
        k = int(k)
        out[i] = (L.orc_glb_partition_hash(k), L.orc_local_partition_hash(k),
                  L.orc_join_hash(k), L.orc_join_hash2(k))
    return out


def glb_partition_hash_np(keys):
    """Vectorised restatement of glb_partition_hash (src/dpu/src/hash.c:117-166)."""
    k = np.asarray(keys, dtype=np.uint64)
    m = np.uint64(0xFFFFFFFF)
    h = (np.uint64(4) + (k & np.uint64(0xFFFF))) & m
    tmp = (((k >> np.uint64(16)) & np.uint64(0xFFFF)) << np.uint64(11)) ^ h
    h = ((h << np.uint64(16)) ^ tmp) & m
    h = (h + (h >> np.uint64(11))) & m
    h = (h ^ (h << np.uint64(3))) & m
    h = (h + (h >> np.uint64(5))) & m
    h = (h ^ (h << np.uint64(4))) & m
    h = (h + (h >> np.uint64(17))) & m
    h = (h ^ (h << np.uint64(25))) & m
    h = (h + (h >> np.uint64(6))) & m
    return h.astype(np.uint32)


def checksum(pairs):
    pairs = _tuples(pairs)
    return int(lib().orc_checksum(_ptr(pairs), pairs.shape[0]))


def sort_pairs(pairs):
    p = _tuples(pairs).copy()
    rc = lib().orc_sort_pairs(_ptr(p), p.shape[0])
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return p


def sort_pairs_mt(pairs, nthreads=None, inplace=False):
    """sort_pairs with threads (the same canonical order); in place when asked."""
    p = _tuples(pairs) if inplace else _tuples(pairs).copy()
    rc = lib().orc_sort_pairs_mt(_ptr(p), p.shape[0], nthreads or os.cpu_count() or 1)
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return p


def generate(n_r, n_s, zipf=0.0, seed=1, nthreads=None):
    """The benchmark relations (R, S) and the checksum of their join, restated
    here so that checkers and CPU arms need no product library. Same values as
    the product's generator."""
    R = np.empty((n_r, 2), dtype=np.uint32)
    S = np.empty((n_s, 2), dtype=np.uint32)
    exp = ctypes.c_uint64(0)
    rc = lib().orc_generate(seed & (2**64 - 1), n_r, n_s, float(zipf), _ptr(R), _ptr(S), ctypes.byref(exp),
                            nthreads or os.cpu_count() or 1)
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return R, S, int(exp.value)


def partition_count(tuples, P, type_=0, rank_sets=1, ranks_per_set=1):
    t = _tuples(tuples)
    hist = np.zeros(P, dtype=np.uint32)
    lib().orc_glb_partition_count(_ptr(t), t.shape[0], type_, P, rank_sets, ranks_per_set, _ptr(hist))
    return hist


def partition_dest(tuples, P, type_=0, rank_sets=1, ranks_per_set=1):
    """Each tuple's global partition as partition_count assigns it (-1 for
    padding, key 0)."""
    t = _tuples(tuples)
    dest = np.empty(t.shape[0], dtype=np.int32)
    lib().orc_glb_partition_dest(_ptr(t), t.shape[0], type_, P, rank_sets, ranks_per_set, _ptr(dest))
    return dest


def chipwise_partition_count(tuples, ranks, rank_sets, bank_set):
    """Histogram of one DPU's S block over the 64 * ranks destinations with
    bank sets (8 ... 64): bank group by hash, DPU in the group by the tuple's
    index, rank set by the index's slot (the chip-wise split)."""
    t = _tuples(tuples)
    hist = np.zeros(64 * ranks, dtype=np.uint32)
    rc = lib().orc_chipwise_partition_count(_ptr(t), t.shape[0], ranks, rank_sets, bank_set, _ptr(hist))
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return hist


def r_dests(key, ranks, rank_sets=1, bank_set=1):
    """The DPUs the reference pipeline sends an R tuple of `key` to (its
    replicas over rank sets and bank-set members included)."""
    out = np.zeros(64 * ranks, dtype=np.int32)
    m = lib().orc_r_dests(int(key), ranks, rank_sets, bank_set, _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


def chipwise_partition_dest(tuples, ranks, rank_sets, bank_set):
    """Each tuple's destination under the chip-wise split (-1 for padding)."""
    t = _tuples(tuples)
    dest = np.empty(t.shape[0], dtype=np.int32)
    rc = lib().orc_chipwise_partition_dest(_ptr(t), t.shape[0], ranks, rank_sets, bank_set, _ptr(dest))
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return dest


def simple_join(R, S, keep_unmatched=False):
    R, S = _tuples(R), _tuples(S)
    out = np.zeros((max(S.shape[0], 1), 2), dtype=np.uint32)
    m = lib().orc_simple_join(_ptr(R), R.shape[0], _ptr(S), S.shape[0], int(keep_unmatched), _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


def simple_join_mt(R, S, keep_unmatched=False, nthreads=None):
    """simple_join with threads: byte-identical output (same pairs, same order)."""
    R, S = _tuples(R), _tuples(S)
    out = np.empty((max(S.shape[0], 1), 2), dtype=np.uint32)
    m = lib().orc_simple_join_mt(_ptr(R), R.shape[0], _ptr(S), S.shape[0], int(keep_unmatched),
                                 nthreads or os.cpu_count() or 1, _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


def refpipe_join(R, S, ranks=1, rank_sets=1, bank_set=1, alg=ALG_PHJ, nthreads=None):
    """The reference pipeline restated: split, partition, replicate, local join."""
    R, S = _tuples(R), _tuples(S)
    nthreads = nthreads or os.cpu_count() or 1
    out = np.empty((max(S.shape[0], 1), 2), dtype=np.uint32)
    m = lib().orc_refpipe_join(_ptr(R), R.shape[0], _ptr(S), S.shape[0], ranks, rank_sets, bank_set, alg,
                               nthreads, _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


def refpipe_dpu_sizes(R, S, ranks=1, rank_sets=1, bank_set=1, nthreads=None):
    R, S = _tuples(R), _tuples(S)
    D = 64 * ranks
    rs = np.zeros(D, dtype=np.int64)
    ss = np.zeros(D, dtype=np.int64)
    rc = lib().orc_refpipe_dpu_sizes(_ptr(R), R.shape[0], _ptr(S), S.shape[0], ranks, rank_sets, bank_set,
                                     nthreads or os.cpu_count() or 1, _ptr(rs), _ptr(ss))
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return rs, ss


def local_partitions(n_r):
    """The local partition count one DPU uses for n_r R tuples (2^bitlen(n_r / 1935))."""
    return int(lib().orc_local_partitions(int(n_r)))


def local_partition(tuples, L):
    """(grouped, offsets): the tuples grouped by local_partition_hash & (L-1),
    input order kept within a group, and the L+1 group starts."""
    t = _tuples(tuples)
    out = np.empty_like(t)
    off = np.zeros(L + 1, dtype=np.int64)
    rc = lib().orc_local_partition(_ptr(t), t.shape[0], L, _ptr(out), _ptr(off))
    if rc:
        raise RuntimeError(ERRORS.get(rc, rc))
    return out, off


def dpu_phj(R, S):
    """One DPU's hash join as the oracle restates it: local partitions, a
    4096-slot linear-probe table per partition, first match per S tuple."""
    R, S = _tuples(R), _tuples(S)
    out = np.empty((max(S.shape[0], 1), 2), dtype=np.uint32)
    m = lib().orc_dpu_phj(_ptr(R), R.shape[0], _ptr(S), S.shape[0], _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


def dpu_smj(R, S):
    """One DPU's sort-merge join as the oracle restates it: S sorted by key,
    each S tuple whose key R holds taking the first such R tuple's payload as
    its key, the others unchanged (all n_s rows)."""
    R, S = _tuples(R), _tuples(S)
    out = np.empty((max(S.shape[0], 1), 2), dtype=np.uint32)
    m = lib().orc_dpu_smj(_ptr(R), R.shape[0], _ptr(S), S.shape[0], _ptr(out))
    if m < 0:
        raise RuntimeError(ERRORS.get(m, m))
    return out[:m]


PRED_NONE, PRED_KEY, PRED_PAYLOAD = 0, 1, 2
PRED_EQ, PRED_LE, PRED_GE, PRED_LT, PRED_GT, PRED_BETWEEN = 0, 1, 2, 3, 4, 5


def select(tuples, field=PRED_KEY, op=PRED_EQ, lo=0, hi=0):
    """The tuples (in input order) whose key (field 1) or payload (field 2)
    passes the predicate, restating the reference's selection predicates
    (src/dpu/include/select.h: PREDINT64's operators ==, <=, >=, <, > at :30-37
    and predi_btw's inclusive range at :44-47) on unsigned 32-bit values."""
    t = _tuples(tuples)
    if field == PRED_NONE:
        return t.copy()
    v = t[:, 0] if field == PRED_KEY else t[:, 1]
    lo, hi = np.uint32(lo), np.uint32(hi)
    keep = {PRED_EQ: v == lo, PRED_LE: v <= lo, PRED_GE: v >= lo, PRED_LT: v < lo, PRED_GT: v > lo,
            PRED_BETWEEN: (lo <= v) & (v <= hi)}[op]
    return t[keep]
