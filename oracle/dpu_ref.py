"""The reference's own DPU join kernels, run on the host.

Test infrastructure only (tests/ imports it, nothing else). ``make -C oracle
ref`` compiles these kernels of yonsei-hpcp/spid-join (src/dpu/src/join/) from
the reference tree, each with the reference's hash.c and the host stand-in for
the DPU runtime in oracle/dpu_host/, into oracle/_ref/dpu_<name>:
  count       glb_partition_count.c
  packet      glb_partition_packet.c
  chipcount   glb_chipwise_partition_count.c
  chippacket  glb_chipwise_partition_packet.c
  bgcount     bg_broadcast_count.c
  bgalign     bg_broadcast_align.c
  lp          a2a_packetwise_srj_local_partition.c
  build       a2a_srj_build.c
  probe       a2a_srj_probe_inner_mt.c
  nl          nested_loop_join.c
  smp         mpsm_join_local_partition.c
  smj         mpsm_join_sort_probe.c
  nbuild      packetwise_no_partitioned_hash_join_build.c
  nprobe      packetwise_no_partitioned_hash_join_probe.c
  finish      finish_join.c
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
RUNNERS = {k: os.path.join(HERE, "_ref", "dpu_" + k)
           for k in ("count", "packet", "chipcount", "chippacket", "bgcount", "bgalign", "build", "probe", "nl", "lp", "smp", "smj", "nbuild", "nprobe",
                     "finish")}
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


def packet_rounds(hist, ranks, packet_size):
    """The packets per destination DPU that the host gives each destination
    rank: the largest count among the rank's 64 DPUs in packets of
    packet_size / 8 tuples, at least one (src/queryHostFunc.cc:1574-1650, for
    one source DPU)."""
    per = packet_size // 8
    top = np.asarray(hist, dtype=np.int64).reshape(ranks, 64).max(axis=1)
    return np.maximum(1, -(-top // per))


def packet_scatter(tuples, ranks, rank_sets=1, dpu_id=0, packet_size=8, bank_set=1, errors=None):
    """The count kernel, then the packet scatter, on one DPU (number dpu_id of
    its rank) holding `tuples`, for 64 * ranks destinations: with bank_set 1
    glb_partition_count.c and glb_partition_packet.c (rank_sets > 1: the
    index-based rank-set split of S), with bank_set 8 ... 64 the chip-wise
    glb_chipwise_partition_count.c and glb_chipwise_partition_packet.c. The
    scatter writes each destination DPU's tuples into its packets: for
    destination rank r a region of packet_rounds[r] rounds of 64 packets, the
    packet of DPU m at slot ((m / 8 - dpu_id / 8) mod 8) + 8 (m mod 8) of each
    round (the rotation that staggers the source DPUs of a bank group).
    Returns, per destination, its packets' slots in order (padding beyond its
    count is checked to be (0, 0)). The kernel's error fields go to `errors`
    (a list) if given; otherwise any nonzero one raises."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n, P = t.shape[0], 64 * ranks
    if P > 2048 or ranks % rank_sets or packet_size not in (8, 16, 32, 64, 128) or not 0 <= dpu_id < 64:
        raise ValueError("64 * ranks <= 2048, rank_sets dividing ranks, packet_size 8..128, dpu_id < 64")
    if bank_set == 1:
        type_, kernel = (0 if rank_sets == 1 else 1), "packet"
        hist, _ = partition_count(t, P, type_, rank_sets, ranks // rank_sets)
    else:
        type_, kernel = 1, "chippacket"
        hist, _ = chipwise_partition_count(t, ranks, rank_sets, bank_set)
    rounds = packet_rounds(hist, ranks, packet_size)
    acc = np.concatenate([[0], np.cumsum(rounds)])
    hist_at = _align(n * 8) + 2048
    ph_at = hist_at + _align(P * 4) + 2048
    res_at = ph_at + _align(ranks * 8) + 2048
    res_bytes = int(acc[-1]) * 64 * packet_size
    mram = np.zeros(res_at + _align(res_bytes) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    _put(mram, hist_at, hist.astype(np.uint32))
    _put(mram, ph_at, rounds.astype(np.int64))
    args = [dpu_id, 0, 0, type_, 0, 0, n, hist_at, ph_at, P, res_at, packet_size, 0, bank_set, rank_sets,
            ranks // rank_sets, JOIN_TYPE_EQUI, 0]
    res, img = launch(kernel, args, mram)
    if errors is not None:
        errors[:] = res[:4]
    elif any(res[:4]):
        raise RuntimeError(f"dpu_{kernel} reported errors {res[:4]}")  # e.g. its counts differ from the count kernel's
    region = img[res_at:res_at + res_bytes].view(np.uint32).reshape(-1, 2)
    per = packet_size // 8
    out = []
    for d in range(P):
        r, m = divmod(d, 64)
        slot = ((m // 8 - dpu_id // 8) % 8) + 8 * (m % 8)
        first = (int(acc[r]) * 64 + slot) * per
        rows = np.concatenate([region[first + k * 64 * per:first + k * 64 * per + per] for k in range(int(rounds[r]))])
        c = int(hist[d])
        if rows[c:].any():
            raise RuntimeError(f"destination {d}: tuples past its count")
        out.append(rows[:c].copy())
    return out


def chipwise_partition_count(tuples, ranks, rank_sets, bank_set):
    """glb_chipwise_partition_count.c on one DPU holding S block `tuples`, for
    64 * ranks destinations, bank sets of `bank_set` (8 ... 64) and `rank_sets`
    rank sets: (histogram, start offsets)."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n, P = t.shape[0], 64 * ranks
    if P > 2048 or bank_set not in (8, 16, 32, 64) or ranks % rank_sets or rank_sets > 256 or \
            P // (bank_set * rank_sets) < 1:
        # its histogram is 2048 words; a bank set of 1 takes the plain count kernel
        raise ValueError("64 * ranks <= 2048, bank_set in 8..64, ranks / rank_sets * 64 >= bank_set")
    info = _align(n * 8) + 2048
    hist = info + _align(P * 4) + 2048
    mram = np.zeros(hist + _align(P * 4) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    args = [0, 1, 0, n, info, hist, P, bank_set, rank_sets, ranks // rank_sets, JOIN_TYPE_EQUI, 0]
    res, img = launch("chipcount", args, mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_chipcount reported errors {res[:4]}")
    return (img[hist:hist + 4 * P].view(np.uint32).copy(), img[info:info + 4 * P].view(np.uint32).copy())


def bg_broadcast_count(tuples, partitions, bank_set):
    """bg_broadcast_count.c on one DPU holding R block `tuples`: (histogram,
    start offsets) over `partitions` bank groups (the reference passes
    ranks per set * 64 / bank_set), by glb_partition_hash."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n, P = t.shape[0], int(partitions)
    if P < 1 or P & (P - 1) or P > 2048:
        raise ValueError("partitions: a power of two up to 2048")
    info = _align(n * 8) + 2048
    hist = info + _align(P * 4) + 2048
    mram = np.zeros(hist + _align(P * 4) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    res, img = launch("bgcount", [0, n, info, hist, P, bank_set, 1, 0], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_bgcount reported errors {res[:4]}")
    return (img[hist:hist + 4 * P].view(np.uint32).copy(), img[info:info + 4 * P].view(np.uint32).copy())


def bg_broadcast_align(tuples, ranks_per_set, bank_set, errors=None):
    """bg_broadcast_count.c, then bg_broadcast_align.c, on one DPU holding R
    block `tuples` with bank sets of `bank_set`: the tuples grouped by their
    ranks_per_set * 64 / bank_set bank groups. Each bank group of rank r gets a
    slot of the size the host gives that rank (its fullest bank group,
    src/queryHostFunc.cc:1731-1770), the slots laid out rank after rank.
    Returns, per bank group, its slot's first `count` tuples (the rest of the
    slot is checked to be (0, 0)). The kernel's error fields go to `errors` (a
    list) if given; otherwise any nonzero one raises."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n = t.shape[0]
    per_rank = 64 // bank_set
    P = ranks_per_set * per_rank
    if bank_set not in (8, 16, 32, 64) or P > 2048:
        raise ValueError("bank_set in 8..64 and ranks_per_set * 64 / bank_set <= 2048")
    hist, _ = bg_broadcast_count(t, P, bank_set)
    slot = hist.astype(np.int64).reshape(ranks_per_set, per_rank).max(axis=1)
    start = np.concatenate([[0], np.cumsum(slot * per_rank)])
    addr = np.array([start[i // per_rank] + (i % per_rank) * slot[i // per_rank] for i in range(P)], dtype=np.int64)
    gh_at = _align(n * 8) + 2048
    ah_at = gh_at + _align(P * 4) + 2048
    res_at = ah_at + _align(ranks_per_set * 4) + 2048
    res_n = int(start[-1])
    mram = np.zeros(res_at + _align(res_n * 8) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    _put(mram, gh_at, hist.astype(np.uint32))
    _put(mram, ah_at, slot.astype(np.uint32))
    res, img = launch("bgalign", [n, P, 0, 0, res_at, gh_at, ah_at, bank_set, 1, 0], mram)
    if errors is not None:
        errors[:] = res[:4]
    elif any(res[:4]):
        raise RuntimeError(f"dpu_bgalign reported errors {res[:4]}")  # e.g. its counts differ from the count kernel's
    region = img[res_at:res_at + 8 * res_n].view(np.uint32).reshape(res_n, 2)
    out = []
    for i in range(P):
        a, c, w = int(addr[i]), int(hist[i]), int(slot[i // per_rank])
        if region[a + c:a + w].any():
            raise RuntimeError(f"bank group {i}: tuples past its count")
        out.append(region[a:a + c].copy())
    return out


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


def range_buckets(elem_range, hist_interval):
    """The number of key-range buckets both sort-merge kernels use:
    elem_range / hist_interval + 1 (mpsm_join_local_partition.c:137,
    mpsm_join_sort_probe.c:281); bucket of a key = min(key / hist_interval,
    buckets - 1)."""
    return int(elem_range) // int(hist_interval) + 1


def probed_buckets(elem_range, hist_interval):
    """Which buckets mpsm_join_sort_probe.c joins (boolean mask). It reads the
    bucket starts in blocks of 512 and walks parts 0..510 of each full block
    (:297) and parts 0..remains-2 of the last (:395), because a part's size is
    start[part+1] - start[part] within the block: bucket 511 of every full
    block and the last bucket are never probed, and their output slots are not
    written."""
    B = range_buckets(elem_range, hist_interval)
    loops, remains = divmod(B, 512)
    b = np.arange(B)
    return (b < loops * 512) & (b % 512 != 511) | (b >= loops * 512) & (b - loops * 512 < remains - 1)


def range_partition(tuples, elem_range, hist_interval):
    """mpsm_join_local_partition.c on one DPU holding `tuples` (key-0 tuples
    are gaps and are dropped): (tuples grouped by key-range bucket, the B
    bucket starts the kernel writes, the non-gap count it returns). Within a
    bucket the order is whichever the tasklets' scatter gave."""
    t = np.ascontiguousarray(tuples, dtype=np.uint32).reshape(-1, 2)
    n = t.shape[0]
    B = range_buckets(elem_range, hist_interval)
    if hist_interval < 1 or not 1 <= B <= 8190:
        # the kernel's histogram is 8192 words and holds B + 1 of them
        raise ValueError("1 <= elem_range / hist_interval + 1 <= 8190")
    sorted_at = _align(n * 8) + 2048
    hist_at = sorted_at + _align(n * 8) + 2048
    mram = np.zeros(hist_at + _align(B * 4) + 2048, dtype=np.uint8)
    _put(mram, 0, t)
    res, img = launch("smp", [elem_range, n, 8, hist_interval, 0, sorted_at, hist_at, 0], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_smp reported errors {res[:4]}")
    m = int(res[4])
    grouped = img[sorted_at:sorted_at + 8 * n].view(np.uint32).reshape(n, 2).copy()
    starts = img[hist_at:hist_at + 4 * B].view(np.uint32).astype(np.int64)
    return grouped, starts, m


def sort_merge(R, S, elem_range, hist_interval):
    """mpsm_join_local_partition.c on R and on S, then mpsm_join_sort_probe.c,
    on one DPU. Each probed S tuple becomes (payload of the R tuple with its
    key, S payload). Returns (rows of the probed buckets in the order the
    kernel wrote them, S tuples of the buckets it leaves unprobed).

    The inputs must keep the kernels on their working path:
      - every key of a probed S bucket is in R (the probe stops its tasklet at
        the first S key R lacks, :226-229, and the others then wait at a
        barrier that never completes);
      - at most 127 tuples of R and of S per bucket (the merge sort writes one
        tuple past a full 128-tuple buffer, :199-202);
      - no probed bucket with S tuples holds exactly one tuple of R or of S
        (the merge sort of one tuple never writes its output buffer, :153-208,
        so the probe would read that buffer's stale contents);
      - B % 512 is 0 or 1, or the last block's B % 512 - 1 buckets are a
        multiple of 12 and all hold S tuples (its loop waits at a barrier once
        per bucket it joins, :477, so every tasklet must join as many)."""
    R = np.ascontiguousarray(R, dtype=np.uint32).reshape(-1, 2)
    S = np.ascontiguousarray(S, dtype=np.uint32).reshape(-1, 2)
    B = range_buckets(elem_range, hist_interval)
    bucket = lambda k: np.minimum(k.astype(np.int64) // hist_interval, B - 1)  # noqa: E731
    rk, sk = R[:, 0][R[:, 0] != 0], S[:, 0][S[:, 0] != 0]
    probed = probed_buckets(elem_range, hist_interval)
    if max(np.bincount(bucket(rk), minlength=B).max(initial=0),
           np.bincount(bucket(sk), minlength=B).max(initial=0)) > 127:
        raise ValueError("more than 127 tuples in a bucket")
    if not np.isin(sk[probed[bucket(sk)]], rk).all():
        raise ValueError("an S key of a probed bucket is not in R")
    r_n, s_n = np.bincount(bucket(rk), minlength=B), np.bincount(bucket(sk), minlength=B)
    if ((s_n > 0) & probed & ((s_n == 1) | (r_n == 1))).any():
        raise ValueError("a probed bucket holds exactly one tuple of R or of S")
    tail = B % 512
    if tail > 1:
        s_tail = np.bincount(bucket(sk), minlength=B)[B - tail:B - 1]
        if (tail - 1) % 12 or not s_tail.all():
            raise ValueError("the last histogram block must hold 12k buckets with S tuples, plus one")
    r_grp, r_start, n_r = range_partition(R, elem_range, hist_interval)
    s_grp, s_start, n_s = range_partition(S, elem_range, hist_interval)
    r_at = 0
    s_at = _align(n_r * 8) + 2048
    rh_at = s_at + _align(n_s * 8) + 2048
    sh_at = rh_at + _align(B * 4) + 2048
    res_at = sh_at + _align(B * 4) + 2048
    mram = np.zeros(res_at + _align(n_s * 8) + 2048, dtype=np.uint8)
    _put(mram, r_at, r_grp[:n_r])
    _put(mram, s_at, s_grp[:n_s])
    _put(mram, rh_at, r_start.astype(np.uint32))
    _put(mram, sh_at, s_start.astype(np.uint32))
    res, img = launch("smj", [elem_range, hist_interval, r_at, s_at, rh_at, sh_at, res_at, 8 * n_r, 8 * n_s], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_smj reported errors {res[:4]}")
    out = img[res_at:res_at + 8 * n_s].view(np.uint32).reshape(n_s, 2)
    keep = probed[bucket(s_grp[:n_s, 0])]
    return out[keep].copy(), s_grp[:n_s][~keep].copy()


def nphj_slots(n_r):
    """The table the reference's host gives one DPU's non-partitioned hash
    join: the power of two just above 16 slots per R tuple
    (src/dpuArgumentJoin.cc:364-376, 389)."""
    return 1 << (int(np.floor(np.log2(16 * max(int(n_r), 1)))) + 1)


def nphj(R, S, slots=None):
    """packetwise_no_partitioned_hash_join_build.c, then
    packetwise_no_partitioned_hash_join_probe.c, on one DPU: one table of
    `slots` 8-byte slots (default nphj_slots(|R|)) over the whole of R, first
    slot join_hash2(key) & (slots - 1). After a collision the kernels step the
    full hash value and reset it to 0 once it reaches `slots` (:143-149 of the
    build), so a collision chain continues at slot 0 (the same sequence in
    build and probe, so the join stays exact). Returns the pairs (R payload, S
    payload) in the order the tasklets wrote them, and the probe's miss count."""
    R = np.ascontiguousarray(R, dtype=np.uint32).reshape(-1, 2)
    S = np.ascontiguousarray(S, dtype=np.uint32).reshape(-1, 2)
    n_r, n_s = R.shape[0], S.shape[0]
    slots = nphj_slots(n_r) if slots is None else int(slots)
    if slots < 32 or slots & (slots - 1) or slots * 8 >= 1 << 31:
        raise ValueError("slots: a power of two, 32 <= slots < 2^28")
    if int((R[:, 0] != 0).sum()) >= slots:
        # the build inserts without a bound: a full table would never finish
        raise ValueError("no more R tuples than table slots - 1")
    r_at = 0
    ht = _align(n_r * 8) + 2048      # the kernels read whole 2 KiB blocks
    s_at = ht + _align(slots * 8) + 2048
    res_at = s_at + _align(n_s * 8) + 2048
    mram = np.zeros(res_at + _align(n_s * 8) + 2048, dtype=np.uint8)
    _put(mram, r_at, R)
    _put(mram, s_at, S)
    res, img = launch("nbuild", [r_at, 8 * n_r, ht, 8 * slots], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_nbuild reported errors {res[:4]}")
    res, img = launch("nprobe", [s_at, 8 * n_s, ht, 8 * slots, res_at], img)
    if any(res[:4]):
        raise RuntimeError(f"dpu_nprobe reported errors {res[:4]}")
    m = int(res[4])
    return img[res_at:res_at + 8 * m].view(np.uint32).reshape(m, 2).copy(), int(res[5])


def nphj_table(R, slots):
    """The table packetwise_no_partitioned_hash_join_build.c leaves after
    inserting R: `slots` rows of (key, payload), key 0 where empty."""
    R = np.ascontiguousarray(R, dtype=np.uint32).reshape(-1, 2)
    n_r = R.shape[0]
    if slots < 32 or slots & (slots - 1) or int((R[:, 0] != 0).sum()) >= slots:
        raise ValueError("slots: a power of two >= 32, above the R tuples")
    ht = _align(n_r * 8) + 2048
    mram = np.zeros(ht + _align(slots * 8) + 2048, dtype=np.uint8)
    _put(mram, 0, R)
    res, img = launch("nbuild", [0, 8 * n_r, ht, 8 * slots], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_nbuild reported errors {res[:4]}")
    return img[ht:ht + 8 * slots].view(np.uint32).reshape(slots, 2).copy()


def finish_join(block, effective):
    """finish_join.c on one DPU whose result block is `block` (m pairs, the
    block's max_bytes = 8 m): the first `effective` pairs are kept and the
    rest of the block becomes (0, 0), so every DPU's block has the common size
    the host transfers."""
    b = np.ascontiguousarray(block, dtype=np.uint32).reshape(-1, 2)
    m = b.shape[0]
    if not 0 <= effective <= m:
        raise ValueError("0 <= effective <= block size")
    at = 2048
    mram = np.full(at + _align(m * 8) + 2048, 0xAB, dtype=np.uint8)
    _put(mram, at, b)
    res, img = launch("finish", [at, 8 * m, 8 * int(effective), 0], mram)
    if any(res[:4]):
        raise RuntimeError(f"dpu_finish reported errors {res[:4]}")
    assert (img[:at] == 0xAB).all() and (img[at + 8 * m:] == 0xAB).all(), "wrote outside its block"
    return img[at:at + 8 * m].view(np.uint32).reshape(m, 2).copy()
