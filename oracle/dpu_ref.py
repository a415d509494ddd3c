"""The reference's own DPU join kernels, run on the host.

Test infrastructure only (tests/ imports it, nothing else): ``make -C oracle
ref`` compiles glb_partition_count.c, a2a_packetwise_srj_local_partition.c,
a2a_srj_build.c, a2a_srj_probe_inner_mt.c and nested_loop_join.c
(src/dpu/src/join/ of yonsei-hpcp/spid-join) from the reference tree, each with
the reference's hash.c and the host stand-in for the DPU runtime in
oracle/dpu_host/, into oracle/_ref/dpu_{count,lp,build,probe,nl}.
One call of a runner is one DPU launch of 12 tasklets over one MRAM image; this
module lays the image out, passes the kernel's arguments and reads its results
back, so that the oracle's restatement of those kernels can be checked against
the kernels themselves.
"""
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RUNNERS = {k: os.path.join(HERE, "_ref", "dpu_" + k) for k in ("count", "build", "probe", "nl", "lp")}
TASKLETS = 12              # NR_TASKLETS of every join kernel
TABLE_BYTES = 32768        # one local partition's hash table (a2a_srj_build.c: 4096 x 8 B)
JOIN_TYPE_EQUI = 1         # include/argument.h
STATUS = {1: "bad runner input", 2: "MRAM access outside the image", 3: "WRAM exhausted"}


def available():
    """Whether the runners were built (they need the reference tree)."""
    return all(os.path.exists(p) for p in RUNNERS.values())


def _align(n, a=2048):
    return (int(n) + a - 1) // a * a


def launch(kernel, args, mram, tasklets=TASKLETS, timeout=120):
    """One DPU launch of `kernel` over the MRAM image `mram` (uint8 array).
    Returns (results, image after the launch)."""
    mram = np.ascontiguousarray(mram, dtype=np.uint8)
    args = [int(a) for a in args]
    msg = (struct.pack("<qq", tasklets, len(args)) + struct.pack("<%dq" % len(args), *args) +
           struct.pack("<q", mram.size) + mram.tobytes())
    out = subprocess.run([RUNNERS[kernel]], input=msg, capture_output=True, check=True, timeout=timeout).stdout
    i = out.index(b"DPUHOST\n") + 8  # the kernels' own prints come first
    status, nres = struct.unpack_from("<qq", out, i)
    i += 16
    if status:
        raise RuntimeError(f"dpu_{kernel}: {STATUS.get(status, status)}")
    res = list(struct.unpack_from("<%dq" % nres, out, i))
    i += 8 * nres
    (nbytes,) = struct.unpack_from("<q", out, i)
    i += 8
    return res, np.frombuffer(out, dtype=np.uint8, count=nbytes, offset=i).copy()


def _put(mram, off, arr):
    b = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    mram[off:off + b.size] = b


def partition_count(tuples, P, type_=0, rank_sets=1, ranks_per_set=1):
    """glb_partition_count.c on one DPU holding `tuples`: (histogram, start
    offsets) of its P global partitions. type_ 0 partitions by the hash (R);
    type_ 1 adds the rank group chosen by the tuple's index (S with rank sets)."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n = t.shape[0]
    if P < 1 or P & (P - 1) or P > 2048:
        raise ValueError("P: a power of two up to 2048")
    info = _align(n * 8) + 2048
    hist = info + _align(P * 4) + 2048
    mram = np.zeros(hist + _align(P * 4) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    args = [0, type_, 0, n, info, hist, P, 1, rank_sets, ranks_per_set, JOIN_TYPE_EQUI, 0]
    res, img = launch("count", args, mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_count reported errors {res[:4]}")
    return (img[hist:hist + 4 * P].view(np.uint32).copy(), img[info:info + 4 * P].view(np.uint32).copy())


def hash_join(r_grouped, r_off, s_grouped, s_off):
    """a2a_srj_build.c, then a2a_srj_probe_inner_mt.c, on one DPU whose R and S
    are laid out in local partitions (offsets r_off / s_off, L+1 entries each,
    as oracle.local_partition gives them). Returns the output pairs in the
    order the kernel wrote them."""
    R = np.ascontiguousarray(r_grouped, dtype=np.uint32).reshape(-1, 2)
    S = np.ascontiguousarray(s_grouped, dtype=np.uint32).reshape(-1, 2)
    L = len(r_off) - 1
    if L < 1 or len(s_off) != L + 1:
        raise ValueError("offsets of the same L >= 1 partitions for R and S")
    if int(np.diff(r_off).max(initial=0)) > TABLE_BYTES // 8:
        # the build kernel inserts without a bound: a fuller table would never finish
        raise ValueError("a local R partition holds more than 4096 tuples")
    n_r, n_s = R.shape[0], S.shape[0]
    r_at = 0
    r_info = r_at + _align(n_r * 8) + 2048
    ht = r_info + _align((L + 4) * 4) + 2048
    s_at = ht + L * TABLE_BYTES
    s_info = s_at + _align(n_s * 8) + 2048
    res_at = s_info + _align((L + 4) * 4) + 2048
    mram = np.zeros(res_at + _align(n_s * 8) + 4096, dtype=np.uint8)
    _put(mram, r_at, R)
    _put(mram, r_info, np.asarray(r_off, dtype=np.uint32))
    _put(mram, s_at, S)
    _put(mram, s_info, np.asarray(s_off, dtype=np.uint32))
    res, img = launch("build", [r_at, 0, ht, r_info, L, n_r, 0], mram)
    if res[2] == 11:  # ERROR_TYPE_2 = 11: the partitions do not add up to R_num
        raise RuntimeError(f"dpu_build: partition sizes do not add up ({res[:4]})")
    res, img = launch("probe", [s_at, 0, ht, s_info, res_at, L, n_s, 0, 0, JOIN_TYPE_EQUI, 0], img)
    if res[1]:  # ERROR_TYPE_1 = 2: an S tuple neither matched nor reached an empty slot
        raise RuntimeError(f"dpu_probe reported errors {res[:4]}")
    m = int(res[4])
    return img[res_at:res_at + 8 * m].view(np.uint32).reshape(m, 2).copy()


def nested_loop(R, S):
    """nested_loop_join.c on one DPU: S rewritten in place, each S tuple whose
    key equals an R key taking that R tuple's payload as its key (R in order,
    blocks of 256 tuples, three blocks at a time), the others unchanged.
    Returns the n_s rewritten S tuples. Quadratic: keep the relations small."""
    R = np.ascontiguousarray(R, dtype=np.uint32).reshape(-1, 2)
    S = np.ascontiguousarray(S, dtype=np.uint32).reshape(-1, 2)
    n_r, n_s = R.shape[0], S.shape[0]
    r_at = 0
    s_at = _align(n_r * 8, 3 * 2048) + 3 * 2048  # whole groups of three R blocks are read
    res_at = s_at + _align(n_s * 8, 12 * 2048) + 12 * 2048
    mram = np.zeros(res_at + _align(n_s * 8, 12 * 2048) + 12 * 2048, dtype=np.uint8)
    _put(mram, r_at, R)
    _put(mram, s_at, S)
    _, img = launch("nl", [r_at, s_at, n_r, n_s, 8, res_at], mram)
    return img[res_at:res_at + 8 * n_s].view(np.uint32).reshape(n_s, 2).copy()


def local_partition(tuples, partitions=0):
    """a2a_packetwise_srj_local_partition.c on one DPU holding `tuples` (key-0
    tuples are gaps and are dropped): (grouped tuples, L + 1 partition starts,
    L). partitions = 0 lets the kernel choose L = 2^bitlen(n / 1935) from its
    non-gap tuples, as it does for R; S passes R's L. At most 512 partitions
    (the kernel writes its start offsets back correctly up to that many)."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n = t.shape[0]
    if partitions > 512:
        raise ValueError("at most 512 local partitions")
    res_at = _align(n * 8) + 2048
    info_at = res_at + _align(n * 8) + 2048
    mram = np.zeros(info_at + 32768 + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    res, img = launch("lp", [0, 0, res_at, info_at, partitions, 0, 1, n, 8, 8, 0, 0], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_lp reported errors {res[:4]}")
    m, L = int(res[4]), int(res[5])
    if L > 512:
        raise RuntimeError("more than 512 local partitions")
    starts = img[info_at:info_at + 4 * L].view(np.uint32).astype(np.int64)
    grouped = img[res_at:res_at + 8 * m].view(np.uint32).reshape(m, 2).copy()
    return grouped, np.append(starts, m), L
