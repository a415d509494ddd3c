"""Deterministic inputs for the golden vectors of the reference's DPU kernels
(dpu_kernel_vectors.json): the same bytes wherever they are rebuilt, from
integer arithmetic alone (a splitmix64 stream), so that the fixture stores
only a case's parameters and the kernels' answers."""
import numpy as np

def _mix(x):
    """The splitmix64 finaliser, elementwise on uint64."""
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def stream(seed, n):
    """n 64-bit values of the splitmix64 sequence that starts at `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)
    return _mix(i)


def relation(seed, n, domain, pad_every=0, payload="index"):
    """n tuples with keys in 1..domain (below 2^31), payloads = the tuple's
    index (or a stream value), and (0, 0) padding at every pad_every-th
    position."""
    v = stream(seed, n)
    keys = (v % np.uint64(domain)).astype(np.uint32) + np.uint32(1)
    pay = np.arange(n, dtype=np.uint32) if payload == "index" else (stream(seed ^ 0x5A5A, n) >> np.uint64(33)).astype(
        np.uint32)
    t = np.stack([keys, pay], 1).astype(np.uint32).reshape(n, 2)
    if pad_every:
        t[::pad_every] = 0
    return t


def fk_pair(seed, n_r, n_s, miss_every=0, dense=False):
    """R: n_r distinct keys with stream payloads, in a seeded order -- the keys
    1..n_r when dense (the sort-merge's range buckets want them), else keys
    spread over 1..2^30 as a DPU receives them after the global partitioning
    (the local partitioning hashes key >> 6, so a dense range would crowd its
    partitions). S: n_s keys drawn from R, every miss_every-th one replaced by
    a key R lacks; payloads = S index."""
    if dense:
        keys = np.arange(1, n_r + 1, dtype=np.uint64)
    else:
        cand = stream(seed + 3, 2 * n_r + 64) % np.uint64(1 << 30) + np.uint64(1)
        _, first = np.unique(cand, return_index=True)
        keys = cand[np.sort(first)][:n_r]
    order = np.argsort(stream(seed, n_r), kind="stable")
    R = np.stack([keys[order].astype(np.uint32), (stream(seed + 1, n_r) >> np.uint64(33)).astype(np.uint32)], 1)
    pick = (stream(seed + 2, n_s) % np.uint64(n_r)).astype(np.int64)
    sk = R[pick, 0].copy()
    if miss_every:
        sk[::miss_every] = np.uint32((1 << 30) + 7)
    S = np.stack([sk, np.arange(n_s, dtype=np.uint32)], 1)
    return np.ascontiguousarray(R, dtype=np.uint32), np.ascontiguousarray(S, dtype=np.uint32)


def checksum(pairs):
    """Order-independent 64-bit digest of (lvalue, rvalue) pairs: the sum of the
    splitmix64 finaliser of (lvalue << 32 | rvalue), the same digest as the
    oracle's and the product's."""
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
    if p.shape[0] == 0:
        return 0
    v = (p[:, 0].astype(np.uint64) << np.uint64(32)) | p[:, 1].astype(np.uint64)
    return int(np.sum(_mix(v), dtype=np.uint64))


def groups_summary(groups):
    """[count, checksum] of each group."""
    return [[int(g.shape[0]), checksum(g)] for g in groups]
