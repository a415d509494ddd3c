"""The oracle against the reference's own DPU join kernels, compiled from the
reference tree as plain C and run on the host (oracle/dpu_ref.py,
oracle/dpu_host/). The kernels, all under src/dpu/src/join/, are these:
  - the global partition counts of glb_partition_count.c,
    glb_chipwise_partition_count.c and bg_broadcast_count.c;
  - the packet scatters of glb_partition_packet.c and
    glb_chipwise_partition_packet.c, and the bank-group R layout of
    bg_broadcast_align.c;
  - the local partitioning of a2a_packetwise_srj_local_partition.c;
  - the hash build and probe of a2a_srj_build.c and a2a_srj_probe_inner_mt.c;
  - the nested loop of nested_loop_join.c;
  - the range partitioning and sort-probe of mpsm_join_local_partition.c and
    mpsm_join_sort_probe.c;
  - the non-partitioned hash join of
    packetwise_no_partitioned_hash_join_{build,probe}.c;
  - the finish kernel of finish_join.c.
Each must give what the oracle's restatement gives on the same inputs. The
runners exist only where the reference tree was present when the oracle was
built; elsewhere these tests are skipped."""
import numpy as np
import pytest

import dpu_ref

pytestmark = pytest.mark.skipif(not dpu_ref.available(), reason="reference DPU kernels not built here")


def _tuples(rng, n, key_hi=2**32):
    return np.stack([rng.integers(0, key_hi, n), np.arange(n)], 1).astype(np.uint32).reshape(n, 2)


@pytest.mark.parametrize("n", [1, 255, 256, 50001])
@pytest.mark.parametrize("P,type_,rank_sets,ranks_per_set",
                         [(64, 0, 1, 1), (1024, 0, 1, 1), (2048, 0, 1, 1), (256, 1, 4, 1), (512, 1, 2, 4),
                          (1024, 1, 16, 1)])
def test_partition_count_kernel(oracle, n, P, type_, rank_sets, ranks_per_set):
    rng = np.random.default_rng(n * 31 + P)
    T = _tuples(rng, n)
    T[::37, 0] = 0  # padding is not counted
    hist, start = dpu_ref.partition_count(T, P, type_, rank_sets, ranks_per_set)
    want = oracle.partition_count(T, P, type_, rank_sets, ranks_per_set)
    assert np.array_equal(hist, want)
    assert np.array_equal(start, (np.cumsum(want) - want).astype(np.uint32))
    assert int(hist.sum()) == int((T[:, 0] != 0).sum())


@pytest.mark.parametrize("n", [1, 256, 20001])
@pytest.mark.parametrize("ranks,rank_sets,dpu_id,packet_size", [(1, 1, 0, 8), (4, 1, 8, 8), (4, 2, 19, 16),
                                                                (8, 4, 63, 64), (32, 1, 40, 128), (16, 16, 7, 8)])
def test_packet_scatter_kernel(oracle, n, ranks, rank_sets, dpu_id, packet_size):
    """glb_partition_count.c, then glb_partition_packet.c with the packet
    counts the host derives from the histogram. The scatter's own check (its
    per-destination counts equal the count kernel's) passes, and every
    destination DPU's packets, read through the rotated layout, hold exactly
    the tuples the oracle sends there, then (0, 0)."""
    rng = np.random.default_rng(n + ranks + dpu_id)
    T = _tuples(rng, n)
    T[::53, 0] = 0
    groups = dpu_ref.packet_scatter(T, ranks, rank_sets, dpu_id, packet_size)
    dest = oracle.partition_dest(T, 64 * ranks, 0 if rank_sets == 1 else 1, rank_sets, ranks // rank_sets)
    assert len(groups) == 64 * ranks
    for d, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == d]))
    assert sum(g.shape[0] for g in groups) == int((T[:, 0] != 0).sum())


def test_packet_rounds_follow_the_fullest_destination():
    """The host sizes a destination rank's packets by its fullest DPU, in
    packets of packet_size / 8 tuples, and gives an empty rank one packet."""
    hist = np.zeros(3 * 64, dtype=np.int64)
    hist[5], hist[64 + 63], hist[64 + 1] = 9, 17, 3
    assert list(dpu_ref.packet_rounds(hist, 3, 8)) == [9, 17, 1]
    assert list(dpu_ref.packet_rounds(hist, 3, 32)) == [3, 5, 1]


@pytest.mark.parametrize("n", [1, 256, 50001])
@pytest.mark.parametrize("ranks,rank_sets,bank_set", [(1, 1, 8), (1, 1, 64), (4, 2, 16), (8, 1, 64), (32, 4, 32),
                                                      (16, 16, 8), (32, 1, 8)])
def test_chipwise_partition_count_kernel(oracle, n, ranks, rank_sets, bank_set):
    """glb_chipwise_partition_count.c (S with bank sets): bank group by hash,
    DPU inside the group by the tuple's index in its 2 KiB block, rank set by
    the index's slot. Its histogram and start offsets equal the oracle's
    chip-wise split."""
    rng = np.random.default_rng(n + ranks * 7 + bank_set)
    T = _tuples(rng, n)
    T[::37, 0] = 0
    hist, start = dpu_ref.chipwise_partition_count(T, ranks, rank_sets, bank_set)
    want = oracle.chipwise_partition_count(T, ranks, rank_sets, bank_set)
    assert np.array_equal(hist, want)
    assert np.array_equal(start, (np.cumsum(want) - want).astype(np.uint32))
    assert int(hist.sum()) == int((T[:, 0] != 0).sum())


@pytest.mark.parametrize("ranks,rank_sets,bank_set", [(1, 1, 64), (4, 2, 16), (32, 4, 8), (64, 2, 8)])
def test_bg_broadcast_count_kernel(oracle, ranks, rank_sets, bank_set):
    """bg_broadcast_count.c (R with bank sets) over the ranks per set * 64 /
    bank_set bank groups the reference passes it: the oracle's hash
    histogram."""
    rng = np.random.default_rng(ranks + bank_set)
    T = _tuples(rng, 30001)
    T[::29, 0] = 0
    P = ranks // rank_sets * 64 // bank_set
    hist, start = dpu_ref.bg_broadcast_count(T, P, bank_set)
    want = oracle.partition_count(T, P, 0)
    assert np.array_equal(hist, want)
    assert np.array_equal(start, (np.cumsum(want) - want).astype(np.uint32))


@pytest.mark.parametrize("ranks_per_set,bank_set", [(1, 64), (1, 8), (4, 16), (32, 8), (8, 32)])
def test_bg_broadcast_align_kernel(oracle, ranks_per_set, bank_set):
    """bg_broadcast_count.c, then bg_broadcast_align.c (R with bank sets) with
    the slot sizes the host derives: each bank group's slot holds exactly the R
    tuples the oracle sends to that bank group, then (0, 0), and the kernel's
    own check (its counts equal the count kernel's) passes."""
    rng = np.random.default_rng(ranks_per_set * 3 + bank_set)
    T = _tuples(rng, 30001, key_hi=2**31)
    T[::29, 0] = 0
    groups = dpu_ref.bg_broadcast_align(T, ranks_per_set, bank_set)
    dest = oracle.partition_dest(T, ranks_per_set * 64 // bank_set, 0)
    for i, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == i]))
    assert sum(g.shape[0] for g in groups) == int((T[:, 0] != 0).sum())


def test_bg_broadcast_align_flags_high_keys(oracle):
    """Like the chip-wise scatter, the align kernel sets ERROR_TYPE_3 = 1 for a
    key of 2^31 or above and still places the tuple in its bank group."""
    rng = np.random.default_rng(78)
    T = _tuples(rng, 4000, key_hi=2**31)
    T[5, 0] = 0xFFFFFFF0
    errors = []
    groups = dpu_ref.bg_broadcast_align(T, 2, 16, errors=errors)
    assert errors == [0, 0, 0, 1]
    dest = oracle.partition_dest(T, 2 * 64 // 16, 0)
    for i, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == i]))


def _join_both(oracle, R, S):
    L = oracle.local_partitions(R.shape[0])
    rg, ro = oracle.local_partition(R, L)
    sg, so = oracle.local_partition(S, L)
    return dpu_ref.hash_join(rg, ro, sg, so), oracle.dpu_phj(R, S)


@pytest.mark.parametrize("n_r,n_s", [(1, 3), (1935, 4000), (20000, 70000), (1 << 15, 1 << 17)])
def test_hash_build_probe_kernels_fk(oracle, n_r, n_s):
    """Unique R keys; S mixes matching keys, keys absent from R and padding:
    one pair per matching S tuple, (R payload, S payload), nothing else."""
    rng = np.random.default_rng(n_r + n_s)
    keys = rng.permutation(np.arange(1, 4 * n_r + 2))[:n_r]
    R = np.stack([keys, rng.integers(0, 2**32, n_r)], 1).astype(np.uint32)
    hit = rng.random(n_s) < 0.8
    S = np.stack([np.where(hit, keys[rng.integers(0, n_r, n_s)], rng.integers(4 * n_r + 2, 2**32, n_s)),
                  np.arange(n_s)], 1).astype(np.uint32)
    S[::53, 0] = 0
    got, restated = _join_both(oracle, R, S)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(restated))
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))


def test_hash_build_probe_kernels_generated(oracle):
    """One DPU's share of the benchmark relations (Zipf 1.0)."""
    R, S, expect = oracle.generate(1 << 15, 1 << 18, 1.0, seed=0x5EED5EED)
    got, restated = _join_both(oracle, R, S)
    assert got.shape == (S.shape[0], 2) and oracle.checksum(got) == expect
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(restated))


def test_hash_build_probe_kernels_repeated_r_keys(oracle):
    """Repeated R keys: the kernels keep every copy and the probe stops at the
    first one on the key's probe sequence, so each S tuple with a key in R
    yields exactly one pair joining equal keys, as in the restatement (which
    copy is first depends on the tasklets' order)."""
    rng = np.random.default_rng(9)
    keys = rng.integers(1, 3000, 12000)
    R = np.stack([keys, np.arange(12000)], 1).astype(np.uint32)
    S = np.stack([rng.integers(1, 6000, 40000), np.arange(40000)], 1).astype(np.uint32)
    got, restated = _join_both(oracle, R, S)
    assert got.shape == restated.shape
    assert np.array_equal(np.sort(got[:, 1]), np.sort(restated[:, 1]))  # the same S tuples matched
    assert np.array_equal(R[got[:, 0], 0], S[got[:, 1], 0])              # each pair joins equal keys


@pytest.mark.parametrize("n_r,n_s", [(1, 5), (256, 257), (700, 3000), (2000, 2500)])
def test_nested_loop_kernel(oracle, n_r, n_s):
    """nested_loop_join.c rewrites S in place: a matched tuple becomes (R
    payload, S payload) from the first equal R key in R order, an unmatched one
    stays. With R payloads that are no R key, that is the oracle's nested-loop
    output, in S order; repeated R keys included."""
    rng = np.random.default_rng(n_r * 3 + n_s)
    keys = rng.integers(1, 3 * n_r + 2, n_r)  # repeats allowed
    R = np.stack([keys, rng.integers(2**31, 2**32, n_r)], 1).astype(np.uint32)
    S = np.stack([np.where(rng.random(n_s) < 0.7, keys[rng.integers(0, n_r, n_s)],
                           rng.integers(3 * n_r + 2, 2**31, n_s)), np.arange(n_s)], 1).astype(np.uint32)
    got = dpu_ref.nested_loop(R, S)
    assert np.array_equal(got, oracle.simple_join(R, S, keep_unmatched=True))


def test_nested_loop_kernel_rewrites_again(oracle):
    """The quirk the oracle's restatement leaves out (and says so): the kernel
    keeps comparing a rewritten key with the later R blocks, so when a matched
    R tuple's payload equals a key further down R the S tuple is rewritten a
    second time. Only those S tuples differ from the single rewrite."""
    R = np.zeros((1000, 2), dtype=np.uint32)
    R[:, 0] = np.arange(1, 1001)
    R[:, 1] = np.arange(1, 1001) + 5000
    R[3] = (4, 999)      # block 0: payload 999 is the key of R[998], three blocks later
    R[998] = (999, 77)
    S = np.array([[4, 0], [5, 1], [999, 2]], dtype=np.uint32)
    got = dpu_ref.nested_loop(R, S)
    want = oracle.simple_join(R, S, keep_unmatched=True)
    assert want.tolist() == [[999, 0], [5005, 1], [77, 2]]
    assert got.tolist() == [[77, 0], [5005, 1], [77, 2]]


@pytest.mark.parametrize("n,gap", [(1, 0), (1936, 0), (30000, 41), (200000, 7)])
def test_local_partition_kernel(oracle, n, gap):
    """a2a_packetwise_srj_local_partition.c: L = 2^bitlen(n / 1935) from the
    non-gap tuples, the start offsets and every partition's tuples equal the
    oracle's local partitioning (the order inside a partition is the tasklets')."""
    rng = np.random.default_rng(n + gap)
    T = np.stack([rng.permutation(np.arange(1, 4 * n + 2))[:n], rng.integers(0, 2**32, n)], 1).astype(np.uint32)
    if gap:
        T[::gap, 0] = 0  # key 0: gaps between packets, dropped
    got, starts, L = dpu_ref.local_partition(T)
    nz = T[T[:, 0] != 0]
    assert L == oracle.local_partitions(nz.shape[0])
    want, off = oracle.local_partition(nz, L)
    assert np.array_equal(starts, off)
    for p in range(L):
        assert np.array_equal(oracle.sort_pairs(got[starts[p]:starts[p + 1]]),
                              oracle.sort_pairs(want[off[p]:off[p + 1]]))


def test_reference_kernels_chained_join(oracle):
    """One DPU's hash join by the reference's kernels alone: local partitioning
    of R (which picks L) and of S (with R's L), then build and probe. The pairs
    equal the oracle's per-DPU join and its independent join."""
    R, S, _ = oracle.generate(60000, 240000, 1.0, seed=7)
    S = S.copy()
    S[::97, 0] = 0  # gaps in S's packets
    rg, ro, L = dpu_ref.local_partition(R)
    sg, so, Ls = dpu_ref.local_partition(S, partitions=L)
    assert Ls == L
    got = dpu_ref.hash_join(rg, ro, sg, so)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.dpu_phj(R, S)))
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))


def _range_bucket(keys, elem_range, interval):
    return np.minimum(keys.astype(np.int64) // interval, dpu_ref.range_buckets(elem_range, interval) - 1)


@pytest.mark.parametrize("n,elem_range,interval,gap", [(1, 64, 64, 0), (5000, 1 << 16, 64, 0),
                                                       (100000, 1 << 16, 64, 13), (70000, 500000, 100, 0)])
def test_range_partition_kernel(n, elem_range, interval, gap):
    """mpsm_join_local_partition.c: the non-gap tuples grouped by key range
    (bucket = min(key / interval, B - 1), so keys past elem_range land in the
    last bucket), the B bucket starts it writes are the exclusive prefix sum of
    the bucket sizes, the slots past the non-gap count are zeroed."""
    rng = np.random.default_rng(n + elem_range)
    keys = rng.integers(1, elem_range + 1, n)
    keys[::101] = rng.integers(elem_range, 2**32, keys[::101].size)  # past the range
    T = np.stack([keys, rng.integers(0, 2**32, n)], 1).astype(np.uint32)
    if gap:
        T[::gap, 0] = 0
    got, starts, m = dpu_ref.range_partition(T, elem_range, interval)
    nz = T[T[:, 0] != 0]
    assert m == nz.shape[0]
    B = dpu_ref.range_buckets(elem_range, interval)
    sizes = np.bincount(_range_bucket(nz[:, 0], elem_range, interval), minlength=B)
    assert np.array_equal(starts, np.cumsum(sizes) - sizes)
    for b in np.flatnonzero(sizes):
        grp = got[starts[b]:starts[b] + sizes[b]]
        assert np.array_equal(oracle_sort(grp), oracle_sort(nz[_range_bucket(nz[:, 0], elem_range, interval) == b]))
    assert not got[m:].any()


def oracle_sort(t):
    return t[np.lexsort((t[:, 1], t[:, 0]))]


def test_sort_probe_bucket_walk():
    """mpsm_join_sort_probe.c joins parts 0..510 of every full block of 512
    bucket starts and parts 0..remains-2 of the last block: bucket 511 of each
    full block and the last bucket are left unprobed."""
    m = dpu_ref.probed_buckets(513 * 64 - 1, 64)  # B = 513
    assert m.size == 513 and m.sum() == 511 and not m[511] and not m[512]
    m = dpu_ref.probed_buckets(1023 * 64, 64)  # B = 1024, no partial block
    assert m.sum() == 1022 and not m[511] and not m[1023]
    m = dpu_ref.probed_buckets(524 * 64, 64)  # B = 525: 12 of the last block's 13
    assert m.sum() == 511 + 12 and m[512:524].all() and not m[524]
    assert dpu_ref.probed_buckets(10, 64).sum() == 0  # B = 1


def _fk_inputs(rng, elem_range, interval, n_s, density=1.0, hot=0):
    """R: a `density` share of the keys 1..elem_range, unique, random payloads;
    S: n_s keys drawn from R (plus `hot` copies of one R key), payloads 0..;
    bucket sizes stay within the kernels' 127-tuple buffers."""
    keys = np.arange(1, elem_range + 1)
    if density < 1.0:
        keys = keys[rng.random(keys.size) < density]
    keys = rng.permutation(keys)
    R = np.stack([keys, rng.integers(0, 2**32, keys.size)], 1).astype(np.uint32)
    sk = np.concatenate([keys[rng.integers(0, keys.size, n_s)], np.full(hot, keys[0])])
    S = np.stack([rng.permutation(sk), np.arange(sk.size)], 1).astype(np.uint32)
    return R, S


@pytest.mark.parametrize("elem_range,interval,n_s,density,hot,gap",
                         [(513 * 64 - 1, 64, 20000, 1.0, 0, 0),     # B = 513
                          (1023 * 64, 64, 40000, 1.0, 40, 0),       # B = 1024, one key 40 more times
                          (524 * 64, 64, 30000, 1.0, 0, 29),        # B = 525: the last block's loop
                          (2047 * 128, 128, 100000, 0.5, 0, 0),     # B = 2048, half the keys in R
                          (4095 * 32, 32, 60000, 1.0, 0, 0)])       # B = 4096
def test_sort_merge_kernels_fk(oracle, elem_range, interval, n_s, density, hot, gap):
    """mpsm_join_local_partition.c on R and on S, then mpsm_join_sort_probe.c:
    on foreign-key inputs (the only ones the probe finishes on) the rows of the
    buckets it probes equal the oracle's per-DPU sort-merge join of those S
    tuples, keys in the same order (S sorted by key within a bucket, buckets by
    range), and the S tuples it leaves unprobed are exactly those of the
    unprobed buckets."""
    rng = np.random.default_rng(elem_range + n_s)
    R, S = _fk_inputs(rng, elem_range, interval, n_s, density, hot)
    if gap:
        R[::gap, 0] = 0  # gaps in both relations' packets; S keeps only keys R still holds
        S = S[np.isin(S[:, 0], R[R[:, 0] != 0, 0])]
        S[::gap, 0] = 0
    rows, unprobed = dpu_ref.sort_merge(R, S, elem_range, interval)
    nz = S[S[:, 0] != 0]
    probed = dpu_ref.probed_buckets(elem_range, interval)[_range_bucket(nz[:, 0], elem_range, interval)]
    want = oracle.dpu_smj(R[R[:, 0] != 0], nz[probed])
    assert rows.shape[0] == want.shape[0] == int(probed.sum())
    assert np.array_equal(rows[:, 0], want[:, 0])
    assert np.array_equal(oracle.sort_pairs(rows), oracle.sort_pairs(want))
    assert np.array_equal(oracle.sort_pairs(rows), oracle.sort_pairs(oracle.simple_join(R, nz[probed])))
    assert np.array_equal(oracle.sort_pairs(unprobed), oracle.sort_pairs(nz[~probed]))


def test_sort_merge_refuses_inputs_the_kernels_cannot_finish():
    """The wrapper refuses, before any launch, the inputs on which the
    reference's sort-probe would stop a tasklet early or overrun a buffer."""
    rng = np.random.default_rng(3)
    R, S = _fk_inputs(rng, 513 * 64 - 1, 64, 20000)
    bad = S.copy()
    bad[0, 0] = 513 * 64 + 5  # last bucket: unprobed, so allowed
    dpu_ref.sort_merge(R, bad, 513 * 64 - 1, 64)
    bad[0, 0] = 2 * 513 * 64  # still the last bucket (clamped)
    dpu_ref.sort_merge(R, bad, 513 * 64 - 1, 64)
    R2 = R[R[:, 0] != 100]
    with pytest.raises(ValueError, match="not in R"):
        dpu_ref.sort_merge(R2, np.array([[100, 0]], dtype=np.uint32), 513 * 64 - 1, 64)
    with pytest.raises(ValueError, match="127"):
        dpu_ref.sort_merge(R, np.array([[R[0, 0], i] for i in range(128)], dtype=np.uint32), 513 * 64 - 1, 64)
    with pytest.raises(ValueError, match="exactly one"):
        dpu_ref.sort_merge(R, S[:1000], 513 * 64 - 1, 64)  # sparse S: buckets of one S tuple
    with pytest.raises(ValueError, match="last histogram block"):
        R3, S3 = _fk_inputs(rng, 600 * 64, 64, 40000)
        dpu_ref.sort_merge(R3, S3, 600 * 64, 64)  # B = 601: the last block's loop joins 88 buckets


@pytest.mark.parametrize("n_r,n_s", [(1, 3), (1000, 5000), (1 << 16, 1 << 18)])
def test_nphj_kernels_fk(oracle, n_r, n_s):
    """packetwise_no_partitioned_hash_join_{build,probe}.c with the table the
    reference's host sizes: unique R keys, S with misses and padding, one pair
    per matching S tuple, equal to the oracle's per-DPU join and the
    independent join."""
    rng = np.random.default_rng(n_r * 7 + n_s)
    keys = rng.permutation(np.arange(1, 4 * n_r + 2))[:n_r]
    R = np.stack([keys, rng.integers(0, 2**32, n_r)], 1).astype(np.uint32)
    hit = rng.random(n_s) < 0.7
    S = np.stack([np.where(hit, keys[rng.integers(0, n_r, n_s)], rng.integers(4 * n_r + 2, 2**32, n_s)),
                  np.arange(n_s)], 1).astype(np.uint32)
    S[::41, 0] = 0
    R[::97, 0] = 0
    got, _ = dpu_ref.nphj(R, S)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.dpu_phj(R, S)))
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))


def test_nphj_kernels_generated(oracle):
    """One DPU's share of the benchmark relations (Zipf 1.0): every S tuple
    joins, and the count and checksum are the generator's answer."""
    R, S, expect = oracle.generate(1 << 16, 1 << 18, 1.0, seed=0x5EED)
    got, _ = dpu_ref.nphj(R, S)
    assert got.shape == (S.shape[0], 2) and oracle.checksum(got) == expect


@pytest.mark.parametrize("slots", [1024, 2048])
def test_nphj_kernels_full_table(oracle, slots):
    """A table at load 1000/1024 and 1000/2048: the long collision chains still
    give the exact join."""
    rng = np.random.default_rng(slots)
    keys = rng.permutation(np.arange(1, 1 << 20))[:1000]
    R = np.stack([keys, np.arange(1000)], 1).astype(np.uint32)
    S = np.stack([np.concatenate([keys, rng.integers(1 << 20, 2**32, 500)]), np.arange(1500)], 1).astype(np.uint32)
    got, miss = dpu_ref.nphj(R, S, slots)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))
    assert miss > 0


def test_nphj_kernels_repeated_r_keys(oracle):
    """Repeated R keys: the build inserts every copy, and the probe stops at
    the first copy on the key's sequence. Each S tuple whose key R holds yields
    one pair joining equal keys (which copy is first depends on the tasklets)."""
    rng = np.random.default_rng(11)
    R = np.stack([rng.integers(1, 3000, 12000), np.arange(12000)], 1).astype(np.uint32)
    S = np.stack([rng.integers(1, 6000, 40000), np.arange(40000)], 1).astype(np.uint32)
    got, _ = dpu_ref.nphj(R, S)
    want = oracle.dpu_phj(R, S)
    assert got.shape == want.shape
    assert np.array_equal(np.sort(got[:, 1]), np.sort(want[:, 1]))
    assert np.array_equal(R[got[:, 0], 0], S[got[:, 1], 0])


def test_nphj_build_chains_restart_at_slot_zero(oracle):
    """The build's collision step adds 1 to the full 32-bit hash and resets it
    to 0 once it reaches the slot count, so a key whose home slot is taken goes
    to the first free slot counting from 0: every slot below a displaced key's
    slot is occupied. (The probe walks the same sequence, so the join is
    exact.)"""
    rng = np.random.default_rng(5)
    slots = 256
    keys = rng.permutation(np.arange(1, 1 << 20))[:200]
    R = np.stack([keys, np.arange(200)], 1).astype(np.uint32)
    table = dpu_ref.nphj_table(R, slots)
    assert np.array_equal(np.sort(table[table[:, 0] != 0, 0]), np.sort(keys))
    h2 = oracle.hashes(table[:, 0])[:, 3].astype(np.int64)
    displaced = [i for i in range(slots) if table[i, 0] and h2[i] >= slots and h2[i] % slots != i]
    assert displaced
    for i in displaced:
        assert (table[:i, 0] != 0).all()


@pytest.mark.parametrize("m,effective", [(1000, 300), (1000, 0), (1000, 1000), (512, 256), (257, 1), (2048, 2047)])
def test_finish_join_kernel(m, effective):
    """finish_join.c keeps a DPU block's first `effective` pairs and turns the
    rest of the block into (0, 0), writing nothing outside it."""
    rng = np.random.default_rng(m + effective)
    block = rng.integers(1, 2**32, (m, 2), dtype=np.uint32)
    out = dpu_ref.finish_join(block, effective)
    assert np.array_equal(out[:effective], block[:effective])
    assert not out[effective:].any()


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 5000])
def test_padded_result_layout_matches_finish_join(spj, n):
    """The facades' padded result layout (FinishJoin with dpu_blocks) is what
    the reference's finish kernel leaves in each of a rank's 64 DPU blocks of
    the common size: the block's pairs, then (0, 0) to the block's end."""
    rng = np.random.default_rng(n)
    pairs = rng.integers(1, 2**32, (n, 2), dtype=np.uint32)
    layout = spj._dpu_blocks(pairs)
    per = layout.shape[0] // 64
    base, extra = divmod(n, 64)
    lo = 0
    for b in range(64):
        cnt = base + (1 if b < extra else 0)
        block = rng.integers(1, 2**32, (per, 2), dtype=np.uint32)  # stale bytes past the pairs
        block[:cnt] = pairs[lo:lo + cnt]
        if per:
            assert np.array_equal(dpu_ref.finish_join(block, cnt), layout[b * per:(b + 1) * per])
        lo += cnt
    assert lo == n


@pytest.mark.parametrize("n", [1, 256, 20001])
@pytest.mark.parametrize("ranks,rank_sets,bank_set,dpu_id,packet_size", [(1, 1, 8, 0, 8), (4, 2, 16, 8, 16),
                                                                         (8, 1, 64, 63, 64), (32, 4, 32, 21, 8),
                                                                         (16, 16, 8, 35, 128)])
def test_chipwise_packet_scatter_kernel(oracle, n, ranks, rank_sets, bank_set, dpu_id, packet_size):
    """glb_chipwise_partition_count.c, then glb_chipwise_partition_packet.c
    (S with bank sets) with the host's packet counts: every destination DPU's
    packets hold exactly the tuples the oracle's chip-wise split sends there,
    then (0, 0), and the kernel reports no error."""
    rng = np.random.default_rng(n + ranks + bank_set + dpu_id)
    T = _tuples(rng, n, key_hi=2**31)
    T[::53, 0] = 0
    groups = dpu_ref.packet_scatter(T, ranks, rank_sets, dpu_id, packet_size, bank_set=bank_set)
    dest = oracle.chipwise_partition_dest(T, ranks, rank_sets, bank_set)
    for d, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == d]))
    assert sum(g.shape[0] for g in groups) == int((T[:, 0] != 0).sum())


def test_chipwise_packet_scatter_flags_high_keys(oracle):
    """The chip-wise scatter sets ERROR_TYPE_3 = 1 for a key of 2^31 or above
    (it tests the key as a signed integer) and scatters the tuple all the
    same, to the oracle's destination."""
    rng = np.random.default_rng(77)
    T = _tuples(rng, 5000, key_hi=2**31)
    T[17, 0] = 0x80000001
    errors = []
    groups = dpu_ref.packet_scatter(T, 4, 1, 0, 8, bank_set=16, errors=errors)
    assert errors == [0, 0, 0, 1]
    dest = oracle.chipwise_partition_dest(T, 4, 1, 16)
    for d, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == d]))


def _split_blocks(T, D):
    """LoadColumn's split of a column over D DPUs (src/query.cc:230-300): padded
    with key-0 tuples to a multiple of D * 8 bytes (a whole extra row when it is
    aligned already) and cut into D equal blocks."""
    per = (T.shape[0] * 8 + (D * 8 - T.shape[0] * 8 % (D * 8))) // 8 // D
    padded = np.zeros((per * D, 2), dtype=np.uint32)
    padded[:T.shape[0]] = T
    return [padded[b * per:(b + 1) * per] for b in range(D)]


def test_reference_kernels_over_one_rank(oracle):
    """The reference's join on one rank of 64 DPUs, every DPU step by its own
    kernels run on the host. Each source DPU's block goes through the count
    kernel and the packet scatter. The exchange hands each destination DPU the
    packets addressed to it (the host's rotate-and-stream only moves them).
    Each destination DPU then runs local partitioning of R, of S with R's
    partition count, the build and the probe. The per-DPU R and S sizes equal
    the oracle's pipeline restatement, and the pairs equal its join and the
    independent join."""
    R, S, expect = oracle.generate(1 << 15, 1 << 17, 1.0, seed=0x5EED0001)
    D = 64
    to_r = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(R, D))]
    to_s = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(S, D))]
    r_in = [np.concatenate([to_r[b][d] for b in range(D)]) for d in range(D)]
    s_in = [np.concatenate([to_s[b][d] for b in range(D)]) for d in range(D)]
    want_r, want_s = oracle.refpipe_dpu_sizes(R, S, ranks=1)
    assert [x.shape[0] for x in r_in] == list(want_r)
    assert [x.shape[0] for x in s_in] == list(want_s)
    pairs = []
    for d in range(D):
        rg, ro, L = dpu_ref.local_partition(r_in[d])
        sg, so, _ = dpu_ref.local_partition(s_in[d], partitions=L)
        pairs.append(dpu_ref.hash_join(rg, ro, sg, so))
    got = np.concatenate(pairs)
    assert got.shape[0] == S.shape[0] and oracle.checksum(got) == expect
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.refpipe_join(R, S, ranks=1)))
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))


def test_reference_kernels_over_two_rank_sets(oracle):
    """The same chain on two ranks in two rank sets (-r 2 -R 2): R is
    partitioned over one rank's 64 DPUs and every rank set receives a copy
    (the host's rank-group copy, src/queryHostFunc.cc:654-776); S is split
    over both rank sets by each tuple's index in its block. The per-DPU sizes
    and the pairs equal the oracle's pipeline restatement."""
    R, S, expect = oracle.generate(1 << 14, 1 << 16, 1.5, seed=0x5EED0002)
    ranks, rank_sets = 2, 2
    D, PR = 64 * ranks, 64 * ranks // rank_sets
    r_in = [[] for _ in range(D)]
    s_in = [[] for _ in range(D)]
    for b, blk in enumerate(_split_blocks(R, D)):
        groups = dpu_ref.packet_scatter(blk, ranks // rank_sets, 1, b % 64)
        for g in range(rank_sets):
            for p in range(PR):
                r_in[g * PR + p].append(groups[p])
    for b, blk in enumerate(_split_blocks(S, D)):
        for d, grp in enumerate(dpu_ref.packet_scatter(blk, ranks, rank_sets, b % 64)):
            s_in[d].append(grp)
    r_in = [np.concatenate(x) for x in r_in]
    s_in = [np.concatenate(x) for x in s_in]
    want_r, want_s = oracle.refpipe_dpu_sizes(R, S, ranks=ranks, rank_sets=rank_sets)
    assert [x.shape[0] for x in r_in] == list(want_r)
    assert [x.shape[0] for x in s_in] == list(want_s)
    pairs = []
    for d in range(D):
        rg, ro, L = dpu_ref.local_partition(r_in[d])
        sg, so, _ = dpu_ref.local_partition(s_in[d], partitions=L)
        pairs.append(dpu_ref.hash_join(rg, ro, sg, so))
    got = np.concatenate(pairs)
    assert got.shape[0] == S.shape[0] and oracle.checksum(got) == expect
    want = oracle.refpipe_join(R, S, ranks=ranks, rank_sets=rank_sets)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))


def test_reference_nested_loop_over_one_rank(oracle):
    """The nested-loop form of the join on one rank of 64 DPUs by the
    reference's kernels: count and packet scatter per source DPU, then
    nested_loop_join.c per destination DPU, which rewrites every S tuple in
    place. The rows (matched ones (R payload, S payload), the others unchanged)
    equal the oracle's nested-loop pipeline. R payloads lie above every key, so
    the kernel's second rewrite of a payload that equals a key cannot occur."""
    rng = np.random.default_rng(0x5EED0003)
    n_r, n_s = 1 << 13, 1 << 15
    keys = rng.permutation(np.arange(1, 4 * n_r))[:n_r]
    R = np.stack([keys, rng.integers(1 << 31, 2**32, n_r)], 1).astype(np.uint32)
    hit = rng.random(n_s) < 0.75
    S = np.stack([np.where(hit, keys[rng.integers(0, n_r, n_s)], rng.integers(4 * n_r, 1 << 30, n_s)),
                  np.arange(n_s)], 1).astype(np.uint32)
    D = 64
    to_r = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(R, D))]
    to_s = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(S, D))]
    rows = []
    for d in range(D):
        r_d = np.concatenate([to_r[b][d] for b in range(D)])
        s_d = np.concatenate([to_s[b][d] for b in range(D)])
        rows.append(dpu_ref.nested_loop(r_d, s_d))
    got = np.concatenate(rows)
    want = oracle.refpipe_join(R, S, ranks=1, alg=oracle.ALG_NL)
    assert got.shape == want.shape == (n_s, 2)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S, keep_unmatched=True)))


def test_reference_nphj_over_one_rank(oracle):
    """The non-partitioned form on one rank of 64 DPUs by the reference's
    kernels: count and packet scatter per source DPU, then the
    non-partitioned build and probe per destination DPU with the table the
    host sizes. The pairs equal the oracle's pipeline for that algorithm."""
    R, S, expect = oracle.generate(1 << 15, 1 << 17, 1.5, seed=0x5EED0004)
    D = 64
    to_r = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(R, D))]
    to_s = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(S, D))]
    pairs = []
    for d in range(D):
        r_d = np.concatenate([to_r[b][d] for b in range(D)])
        s_d = np.concatenate([to_s[b][d] for b in range(D)])
        pairs.append(dpu_ref.nphj(r_d, s_d)[0])
    got = np.concatenate(pairs)
    assert got.shape[0] == S.shape[0] and oracle.checksum(got) == expect
    want = oracle.refpipe_join(R, S, ranks=1, alg=oracle.ALG_NPHJ)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))


def test_reference_sort_merge_over_one_rank(oracle):
    """The sort-merge form on one rank of 64 DPUs by the reference's kernels:
    count and packet scatter per source DPU, then per destination DPU the
    range partitioning and the sort-probe with the arguments the reference's
    host passes (elem_range = |R| keys 1..|R|, hist_interval = 64 DPUs * 64,
    src/queryDpuFunc.cc:538-555, src/dpuArgumentJoin.cc:517, 566-567). |R| = 12 *
    4096 gives 13 buckets, of which the sort-probe joins the first 12 (the
    last, key 49152 alone, it leaves unprobed). The probed rows equal the
    oracle's sort-merge pipeline's rows for those S tuples."""
    rng = np.random.default_rng(0x5EED0005)
    n_r = n_s = 12 * 4096
    R = np.stack([rng.permutation(np.arange(1, n_r + 1)), rng.integers(0, 2**32, n_r)], 1).astype(np.uint32)
    S = np.stack([rng.integers(1, n_r + 1, n_s), np.arange(n_s)], 1).astype(np.uint32)
    D = 64
    to_r = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(R, D))]
    to_s = [dpu_ref.packet_scatter(blk, 1, 1, b) for b, blk in enumerate(_split_blocks(S, D))]
    rows, unprobed = [], []
    for d in range(D):
        r_d = np.concatenate([to_r[b][d] for b in range(D)])
        s_d = np.concatenate([to_s[b][d] for b in range(D)])
        got, skipped = dpu_ref.sort_merge(r_d, s_d, n_r, 64 * 64)
        rows.append(got)
        unprobed.append(skipped)
    rows, unprobed = np.concatenate(rows), np.concatenate(unprobed)
    assert np.array_equal(np.sort(unprobed[:, 1]), np.sort(S[S[:, 0] == n_r, 1]))
    want = oracle.refpipe_join(R, S, ranks=1, alg=oracle.ALG_SMJ)
    probed = ~np.isin(want[:, 1], unprobed[:, 1])
    assert rows.shape[0] == int(probed.sum()) == n_s - unprobed.shape[0]
    assert np.array_equal(oracle.sort_pairs(rows), oracle.sort_pairs(want[probed]))


@pytest.mark.parametrize("ranks,rank_sets,bank_set", [(1, 1, 8), (2, 2, 16)])
def test_reference_kernels_with_bank_sets(oracle, ranks, rank_sets, bank_set):
    """The join with bank sets (-B) by the reference's kernels, except the
    host's chip-wise broadcast of R. R: bank-group count and align per source
    DPU; each bank group's tuples go to the DPUs the oracle's pipeline sends
    them to (the broadcast itself runs in the host's transfer code). S: the
    chip-wise count and packet scatter. Then local partitioning, build and
    probe per DPU. Every S tuple finds its R tuple on the DPU the reference's
    own S routing chose, so the per-DPU sizes and the pairs equal the oracle's
    pipeline, and the count and checksum its generator's answer."""
    R, S, expect = oracle.generate(1 << 14, 1 << 16, 1.0, seed=0x5EED0006 + bank_set)
    D, rps = 64 * ranks, ranks // rank_sets
    r_in = [[] for _ in range(D)]
    s_in = [[] for _ in range(D)]
    for blk in _split_blocks(R, D):
        for grp in dpu_ref.bg_broadcast_align(blk, rps, bank_set):
            if grp.shape[0]:
                for d in oracle.r_dests(grp[0, 0], ranks, rank_sets, bank_set):
                    r_in[d].append(grp)
    for b, blk in enumerate(_split_blocks(S, D)):
        for d, grp in enumerate(dpu_ref.packet_scatter(blk, ranks, rank_sets, b % 64, bank_set=bank_set)):
            s_in[d].append(grp)
    r_in = [np.concatenate(x) if x else np.zeros((0, 2), np.uint32) for x in r_in]
    s_in = [np.concatenate(x) for x in s_in]
    want_r, want_s = oracle.refpipe_dpu_sizes(R, S, ranks=ranks, rank_sets=rank_sets, bank_set=bank_set)
    assert [x.shape[0] for x in r_in] == list(want_r)
    assert [x.shape[0] for x in s_in] == list(want_s)
    pairs = []
    for d in range(D):
        rg, ro, L = dpu_ref.local_partition(r_in[d])
        sg, so, _ = dpu_ref.local_partition(s_in[d], partitions=L)
        pairs.append(dpu_ref.hash_join(rg, ro, sg, so))
    got = np.concatenate(pairs)
    assert got.shape[0] == S.shape[0] and oracle.checksum(got) == expect
    want = oracle.refpipe_join(R, S, ranks=ranks, rank_sets=rank_sets, bank_set=bank_set)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))


def test_local_partition_kernel_rejects_high_keys():
    """The local partitioning kernel tests a key as a signed integer: at a key
    of 2^31 or above it sets ERROR_TYPE_1 = 2 and stops reading its block, so
    the reference's path carries keys below 2^31 only (the chip-wise scatter
    and the bank-group align kernel flag the same keys)."""
    T = np.array([[5, 1], [0x80000000, 2], [7, 3]], dtype=np.uint32)
    with pytest.raises(RuntimeError, match=r"\[0, 2, 0, 0\]"):
        dpu_ref.local_partition(T)
    got, starts, L = dpu_ref.local_partition(T[[0, 2]])
    assert L == 1 and starts.tolist() == [0, 2]
