"""GPU parity: the CUDA join through the C ABI against the oracle on the same
seeded inputs -- exact pair multisets (canonical sort), counts and checksums."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import main_cc_tables

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def run_instance(spj, R, S, ranks=1, rank_sets=1, **design_kw):
    inst = spj.JoinInstance(ranks, rank_sets, ranks // rank_sets)
    inst.LoadColumn(R, R.shape[0], "left")
    inst.LoadColumn(S, S.shape[0], "right")
    d = spj.make_design(rank_num=ranks, rank_set=rank_sets, **design_kw)
    inst.PrepareJoin(d)
    inst.StartJoin(d)
    res = inst.FinishJoin()
    logs = inst.RecordLogs()
    inst.close()
    return res, logs


def same_multiset(oracle, a, b):
    return a.shape == b.shape and np.array_equal(oracle.sort_pairs(a), oracle.sort_pairs(b))


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "kat_main_cc.json")))["cases"],
                         ids=lambda c: f"N{c['N']}x{c['ratio']}")
def test_kat_main_cc(spj, oracle, case):
    R, S = main_cc_tables(case["N"], case["ratio"])
    res, _ = run_instance(spj, R, S)
    out = res.pairs()
    assert out.shape[0] == case["n_pairs"]
    assert oracle.checksum(out) == case["checksum"]
    assert sum(res.byte_sizes) == 8 * case["n_pairs"]


@pytest.mark.parametrize("bits", [0, 11])  # 0: the planner's plan (non-partitioned for small R), 11: partitioned
@pytest.mark.parametrize("zipf", [0.0, 1.0, 1.5])
@pytest.mark.parametrize("n_r,ratio", [(1 << 10, 2), (1 << 16, 4), (100003, 3), (1 << 20, 2)])
def test_generated_joins(spj, oracle, zipf, n_r, ratio, bits):
    R, S, expect = spj.generate_host(n_r, n_r * ratio, zipf, seed=n_r + int(10 * zipf))
    res, logs = run_instance(spj, R, S, radix_bits=bits)
    assert logs["join_alg"] == (1 if bits == 0 else 0)
    out = res.pairs()
    assert out.shape[0] == S.shape[0]
    assert oracle.checksum(out) == expect
    assert same_multiset(oracle, out, oracle.simple_join(R, S))
    assert logs["n_pairs"] == S.shape[0]


@pytest.mark.parametrize("layout", [(1, 1, 1, 0), (4, 4, 1, 1), (16, 4, 4, 1), (4, 1, 16, 1), (4, 1, 4, 0)])
def test_replication_groups_bit_exact(spj, oracle, layout):
    ranks, rsets, bset, mode = layout
    R, S, expect = spj.generate_host(1 << 17, 1 << 19, 1.5, seed=31)
    # an explicit fan-out keeps the partitioned join (the planner would run this
    # small R without partitions)
    res, logs = run_instance(spj, R, S, ranks=ranks, rank_sets=rsets, bank_set=bset, skew_mode=mode, radix_bits=11)
    out = res.pairs()
    assert out.shape[0] == S.shape[0] and oracle.checksum(out) == expect


@pytest.mark.parametrize("bits,slots", [(6, 4096), (9, 2048), (12, 12288), (14, 12288), (3, 28000)])
def test_tuning_variants(spj, oracle, bits, slots):
    R, S, expect = spj.generate_host(1 << 15, 1 << 17, 1.0, seed=bits)
    res, logs = run_instance(spj, R, S, radix_bits=bits, table_slots=slots, unit_tuples=4096)
    out = res.pairs()
    assert oracle.checksum(out) == expect and out.shape[0] == S.shape[0]
    assert logs["radix_bits"] == bits


@pytest.mark.parametrize("bits", [0, 9])
def test_non_fk_and_key_zero(spj, oracle, bits):
    rng = np.random.default_rng(5)
    R = np.stack([rng.permutation(np.arange(1, 50001)), rng.integers(0, 2**32, 50000)], 1).astype(np.uint32)
    R[::97, 0] = 0
    S = np.stack([rng.integers(0, 100000, 300001), np.arange(300001)], 1).astype(np.uint32)
    res, _ = run_instance(spj, R, S, radix_bits=bits)
    assert same_multiset(oracle, res.pairs(), oracle.simple_join(R, S))


@pytest.mark.parametrize("bits", [0, 9])
def test_duplicate_r_keys_one_match_each(spj, oracle, bits):
    rng = np.random.default_rng(6)
    keys = rng.integers(1, 2000, 40000)
    R = np.stack([keys, np.arange(40000)], 1).astype(np.uint32)
    S = np.stack([rng.integers(1, 4000, 100000), np.arange(100000)], 1).astype(np.uint32)
    out = run_instance(spj, R, S, radix_bits=bits)[0].pairs()
    present = np.zeros(4001, bool)
    present[keys] = True
    assert out.shape[0] == int(present[S[:, 0]].sum())        # one match per S tuple with a key in R
    assert np.array_equal(np.sort(out[:, 1]), np.sort(S[present[S[:, 0]], 1]))
    assert np.array_equal(R[out[:, 0], 0], S[out[:, 1], 0])   # each pair joins equal keys


@pytest.mark.parametrize("bits", [0, 9])
@pytest.mark.parametrize("nr,ns", [(0, 10), (10, 0), (0, 0), (1, 1), (3, 5), (1, 100000), (100000, 1)])
def test_edge_sizes(spj, oracle, nr, ns, bits):
    rng = np.random.default_rng(nr * 7 + ns)
    R = np.stack([rng.permutation(np.arange(1, nr + 1)), np.arange(nr)], 1).astype(np.uint32).reshape(nr, 2)
    S = np.stack([rng.integers(1, max(nr, 1) + 1, ns), np.arange(ns)], 1).astype(np.uint32).reshape(ns, 2)
    res, _ = run_instance(spj, R, S, radix_bits=bits)
    assert same_multiset(oracle, res.pairs(), oracle.simple_join(R, S))


def test_partition_histogram_matches_count_kernel(spj, oracle):
    import torch
    R, S, _ = spj.generate_host(1 << 18, 1 << 18, 1.0, seed=4)
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    for bits in (6, 10, 14):
        hist = torch.zeros(1 << bits, dtype=torch.int32, device="cuda")
        spj.check(spj.lib().spj_partition_histogram(dR.data_ptr(), R.shape[0], bits, hist.data_ptr(), None))
        torch.cuda.synchronize()
        assert np.array_equal(hist.cpu().numpy().view(np.uint32), oracle.partition_count(R, 1 << bits))


def test_device_plan_full_size_property(spj):
    """|R| = 2^24, |S| = 2^26 Zipf 1.0 on device: pair count and checksum equal the
    generator's exact answer (a size-independent property; the oracle is not needed)."""
    import torch
    n_r, n_s = 1 << 24, 1 << 26
    dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
    dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
    exp = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_generate_device(77, n_r, n_s, 1.0, dR.data_ptr(), dS.data_ptr(), exp.data_ptr(), None))
    plan = spj.Plan(n_r, n_s, spj.make_design(rank_num=1))
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):  # twice: the plan is reusable
        plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n_out.data_ptr(), 0)
        spj.check(spj.lib().spj_checksum_device(out.data_ptr(), n_out.data_ptr(), cs.data_ptr(), None))
        torch.cuda.synchronize()
        st = plan.stats()
        assert int(n_out.item()) == n_s
        assert int(cs.item()) == int(exp.item())
        assert st["n_pairs"] == n_s
    plan.close()


def test_device_generator_matches_host(spj):
    import torch
    n_r, n_s = 1 << 16, 1 << 18
    for z in (0.0, 1.0):
        R, S, exp_h = spj.generate_host(n_r, n_s, z, seed=123)
        dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
        dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
        exp = torch.zeros(1, dtype=torch.int64, device="cuda")
        spj.check(spj.lib().spj_generate_device(123, n_r, n_s, z, dR.data_ptr(), dS.data_ptr(), exp.data_ptr(),
                                                None))
        torch.cuda.synchronize()
        assert np.array_equal(dR.cpu().numpy().view(np.uint32), R)
        diff = (dS.cpu().numpy().view(np.uint32) != S).any(axis=1).sum()
        if z == 0.0:
            assert diff == 0 and int(exp.item()) & (2**64 - 1) == exp_h
        else:
            assert diff <= 2  # libm and CUDA double exp/log may differ in the last ulp


ALGS = ["phj", "nphj", "smj", "nl"]


def alg_design(alg):
    """The design keys of a local-join algorithm: the hash join with an explicit
    fan-out stays partitioned (the planner runs a small R alone without
    partitions)."""
    return dict(join_alg=alg, radix_bits=11) if alg == "phj" else dict(join_alg=alg)


@pytest.mark.parametrize("alg", ALGS)
@pytest.mark.parametrize("zipf", [0.0, 1.0, 1.5])
def test_algorithms_on_fk_joins(spj, oracle, alg, zipf):
    R, S, expect = spj.generate_host(1 << 16, 1 << 18, zipf, seed=77 + int(zipf * 10))
    res, _ = run_instance(spj, R, S, **alg_design(alg))
    out = res.pairs()
    assert out.shape[0] == S.shape[0] and oracle.checksum(out) == expect
    assert same_multiset(oracle, out, oracle.simple_join(R, S))


@pytest.mark.parametrize("alg", ALGS)
def test_algorithms_non_fk_semantics(spj, oracle, alg):
    """PHJ/NPHJ drop unmatched S tuples; SMJ/NL rewrite S in place and keep them."""
    rng = np.random.default_rng(8)
    R = np.stack([rng.permutation(np.arange(1, 30001)), rng.integers(0, 2**32, 30000)], 1).astype(np.uint32)
    R[::101, 0] = 0
    S = np.stack([rng.integers(0, 60000, 200003), np.arange(200003)], 1).astype(np.uint32)
    out = run_instance(spj, R, S, **alg_design(alg))[0].pairs()
    keep = alg in ("smj", "nl")
    assert same_multiset(oracle, out, oracle.simple_join(R, S, keep_unmatched=keep))


@pytest.mark.parametrize("alg", ALGS)
def test_algorithms_duplicate_r_keys(spj, alg):
    rng = np.random.default_rng(9)
    keys = np.concatenate([np.arange(1, 3000), rng.integers(1, 3000, 30000 - 2999)])  # every key present
    rng.shuffle(keys)
    R = np.stack([keys, np.arange(30000)], 1).astype(np.uint32)
    S = np.stack([rng.integers(1, 3000, 90000), np.arange(90000)], 1).astype(np.uint32)
    out = run_instance(spj, R, S, **alg_design(alg))[0].pairs()
    assert out.shape[0] == S.shape[0]  # every S key occurs in R here
    assert np.array_equal(np.sort(out[:, 1]), np.arange(90000, dtype=np.uint32))
    assert np.array_equal(R[out[:, 0], 0], S[out[:, 1], 0])


def test_config3_sweep_all_bit_exact(spj, oracle):
    """Config-3 shape at 1/512 scale (|R| = 2^17, |S| = 2^20, Zipf 1.5): hash, sort-merge,
    nested-loop and non-partitioned joins, and replication groups of 1, 4 and 16 CTAs,
    all give the same multiset."""
    R, S, expect = spj.generate_host(1 << 17, 1 << 20, 1.5, seed=3)
    ref = oracle.sort_pairs(oracle.simple_join(R, S))
    variants = [alg_design(a) for a in ALGS]
    variants += [dict(join_alg="phj", skew_mode=1, ranks=g, rank_sets=g) for g in (1, 4, 16)]
    for v in variants:
        v = dict(v)
        ranks, rsets = v.pop("ranks", 1), v.pop("rank_sets", 1)
        out = run_instance(spj, R, S, ranks=ranks, rank_sets=rsets, **v)[0].pairs()
        assert oracle.checksum(out) == expect, v
        assert np.array_equal(oracle.sort_pairs(out), ref), v


@pytest.mark.parametrize("alg", ALGS)
@pytest.mark.parametrize("nr,ns", [(0, 10), (10, 0), (1, 1), (3, 5), (7, 100000)])
def test_algorithms_edge_sizes(spj, oracle, alg, nr, ns):
    rng = np.random.default_rng(nr * 13 + ns)
    R = np.stack([rng.permutation(np.arange(1, nr + 1)), np.arange(nr)], 1).astype(np.uint32).reshape(nr, 2)
    S = np.stack([rng.integers(1, nr + 3, ns), np.arange(ns)], 1).astype(np.uint32).reshape(ns, 2)
    out = run_instance(spj, R, S, **alg_design(alg))[0].pairs()
    assert same_multiset(oracle, out, oracle.simple_join(R, S, keep_unmatched=alg in ("smj", "nl")))


@pytest.mark.parametrize("alg", [0, 1, 2, 3])
def test_host_columns_joined_in_overlapped_slices(spj, oracle, alg):
    # |S| above 2^26 host tuples: the instance joins S in slices (copy-in,
    # join and copy-out of different slices overlap); the first slice is
    # shorter and has a plan of its own, and every slice after the first of
    # its plan reuses R's partitions. The union of the slices must be the whole
    # join, twice in a row, and again after both columns are replaced by new
    # ones of the same sizes (the plans are reused; R is partitioned anew).
    n_r, n_s = 1 << 22, (1 << 26) + (1 << 20) + 7
    R, S, expect = spj.generate_host(n_r, n_s, 1.0, seed=77)
    inst = spj.JoinInstance(4, 4, 1)
    inst.LoadColumn(R, n_r, "left")
    inst.LoadColumn(S, n_s, "right")
    d = spj.make_design(rank_num=4, rank_set=4, join_alg=alg)
    inst.PrepareJoin(d)
    for _ in range(2):
        inst.StartJoin(d)
        out = inst.FinishJoin().pairs()
        assert out.shape == (n_s, 2)
        assert oracle.checksum(out) == expect
    logs = inst.RecordLogs()
    assert logs["n_pairs"] == n_s
    R2, S2, expect2 = spj.generate_host(n_r, n_s, 0.5, seed=78)
    inst.LoadColumn(R2, n_r, "left")
    inst.LoadColumn(S2, n_s, "right")
    inst.PrepareJoin(d)
    inst.StartJoin(d)
    out = inst.FinishJoin().pairs()
    inst.close()
    assert out.shape == (n_s, 2) and oracle.checksum(out) == expect2


def test_start_after_loading_columns_of_other_sizes(spj, oracle):
    # StartJoin after LoadColumn without PrepareJoin: the instance prepares for
    # the new sizes itself. A sliced S whose size is not a multiple of the slice
    # (key-0 padding in the last slice), then an unsliced one, then the first
    # sizes again: every join exact.
    inst = spj.JoinInstance(1, 1, 1)
    d = spj.make_design(rank_num=1)
    for i, (n_r, n_s, z) in enumerate([(1 << 16, (1 << 24) + 5, 1.0), (1 << 15, 3 << 20, 0.0),
                                       (1 << 16, (1 << 24) + 5, 1.2)]):
        R, S, expect = spj.generate_host(n_r, n_s, z, seed=90 + i)
        inst.LoadColumn(R, n_r, "left")
        inst.LoadColumn(S, n_s, "right")
        if i == 0:
            inst.PrepareJoin(d)
        inst.StartJoin(d)
        out = inst.FinishJoin().pairs()
        assert out.shape == (n_s, 2) and oracle.checksum(out) == expect
    inst.close()



@pytest.mark.parametrize("n_r,n_s,seed", [(1 << 20, 1 << 22, 0x5EED5EED), (100003, 777777, 5)])
def test_oracle_generator_equals_device_generator(spj, oracle, n_r, n_s, seed):
    """The CPU arms of the benchmark make their inputs with the oracle's copy of
    the generator: R and uniform S equal the device generator's bytes, and the
    expected checksums agree (Zipf S is compared with the product's host
    generator on the CPU: its exp/log are the host's)."""
    import torch
    dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
    dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_generate_device(seed, n_r, n_s, 0.0, dR.data_ptr(), dS.data_ptr(), e.data_ptr(), None))
    torch.cuda.synchronize()
    R, S, expect = oracle.generate(n_r, n_s, 0.0, seed=seed)
    assert np.array_equal(dR.cpu().numpy().view(np.uint32), R)
    assert np.array_equal(dS.cpu().numpy().view(np.uint32), S)
    assert int(e.item()) & (2**64 - 1) == expect


@pytest.mark.parametrize("n_r,alg_run", [(1 << 22, 1), ((1 << 22) + 1, 0)])
def test_planner_non_partitioned_up_to_2_22(spj, oracle, n_r, alg_run):
    """A hash join planned alone runs without partitions up to |R| = 2^22 (its
    table fits half of L2), partitioned above; the direct probe (no work units,
    dense output) gives the oracle's pairs, padding and misses included."""
    import torch
    n_s = (1 << 23) + 5
    R, S, _ = spj.generate_host(n_r, n_s, 1.2, seed=71)
    S = S.copy()
    S[::101, 0] = 0                      # padding
    S[5::103, 0] = np.uint32(0xFFFFFFF0)  # keys absent from R
    plan = spj.Plan(n_r, n_s, spj.make_design(rank_num=1))
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):  # the second execution reuses the cleared table
        n.zero_()
        plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n.data_ptr())
        torch.cuda.synchronize()
        st = plan.stats()
        assert st["join_alg"] == alg_run
        k = int(n.item())
        assert k == st["n_pairs"]
        got = out[:k].cpu().numpy().view(np.uint32)
        assert same_multiset(oracle, got, oracle.simple_join_mt(R, S))
    plan.close()


def _join_hash2_np(keys):
    """join_hash2 of the reference (src/dpu/src/hash.c:85-112), vectorised."""
    k = np.asarray(keys, dtype=np.uint64)
    m = np.uint64(0xFFFFFFFF)
    h = np.zeros_like(k)
    for b in range(4):
        h = (h + ((k >> np.uint64(8 * b)) & np.uint64(0xFF))) & m
        h = (h + (h << np.uint64(10))) & m
        h = h ^ (h >> np.uint64(6))
    h = (h + (h << np.uint64(3))) & m
    h = h ^ (h >> np.uint64(11))
    h = (h + (h << np.uint64(15))) & m
    return h.astype(np.uint32)


def test_non_partitioned_clustered_keys(spj, oracle):
    """Every R key of a non-partitioned join alone has its home slot in the
    first quarter of the table (12000 keys for 8192 slots), so the linear probe
    runs far past the home slots and wraps their cluster into the rest of the
    table; the join must still equal the oracle's, repeated keys and misses
    included."""
    import torch
    cand = np.arange(1, 200000, dtype=np.uint32)
    assert oracle.hashes(cand[:4])[:, 3].tolist() == _join_hash2_np(cand[:4]).tolist()
    home = _join_hash2_np(cand) & np.uint32((1 << 15) - 1)  # the planner's table: 2^15 slots for 12000 R
    keys = cand[(home >> 13) == 0][:12000]
    assert keys.shape[0] == 12000
    rng = np.random.default_rng(17)
    R = np.stack([keys, rng.choice(2**31, 12000, replace=False)], 1).astype(np.uint32)  # distinct payloads
    R[::50, 0] = R[1::50, 0]  # some repeated keys (one match per S tuple)
    S = np.stack([np.concatenate([keys[rng.integers(0, 12000, 30000)], rng.integers(200000, 2**31, 5000)]),
                  np.arange(35000)], 1).astype(np.uint32)
    plan = spj.Plan(R.shape[0], S.shape[0], spj.make_design(rank_num=1))
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n.data_ptr())
        torch.cuda.synchronize()
        assert plan.stats()["join_alg"] == 1
        got = out[:int(n.item())].cpu().numpy().view(np.uint32)
        want = oracle.simple_join(R, S)
        assert got.shape == want.shape
        assert np.array_equal(np.sort(got[:, 1]), np.sort(want[:, 1]))  # the same S tuples matched
        by_pay = np.argsort(R[:, 1])                                     # R payloads are distinct
        r_of = by_pay[np.searchsorted(R[by_pay, 1], got[:, 0])]
        assert np.array_equal(R[r_of, 1], got[:, 0])                     # the pair's R payload exists
        assert np.array_equal(R[r_of, 0], S[got[:, 1], 0])               # and joins equal keys
    plan.close()


def test_finish_join_dpu_block_layout(spj, oracle):
    """FinishJoin(dpu_blocks=True): per rank 64 blocks of one size with (0, 0)
    padding, the reference's transfer layout; its non-padding pairs are the
    join (the reference driver's inputs have no (0, 0) pair of their own)."""
    R, S = main_cc_tables(100003, 3)
    inst = spj.JoinInstance(4, 2, 2)
    inst.LoadColumn(R, R.shape[0], "left")
    inst.LoadColumn(S, S.shape[0], "right")
    d = spj.make_design(rank_num=4, rank_set=2)
    inst.PrepareJoin(d)
    inst.StartJoin(d)
    plain = inst.FinishJoin()
    inst.StartJoin(d)
    res = inst.FinishJoin(dpu_blocks=True)
    inst.close()
    assert len(res.buffers) == 4
    # which pairs a rank holds differs between executions (the output order is
    # free); each rank's count does not
    for buf, size, ref in zip(res.buffers, res.byte_sizes, plain.buffers):
        assert size == 8 * buf.shape[0] and buf.shape[0] % 64 == 0
        assert buf.shape[0] // 64 == -(-ref.shape[0] // 64)
        blocks = buf.reshape(64, -1, 2)
        filled = ((blocks[:, :, 0] != 0) | (blocks[:, :, 1] != 0)).sum(1)
        assert filled.sum() == ref.shape[0] and filled.max() - filled.min() <= 1  # dealt evenly
    got = np.concatenate([b[(b[:, 0] != 0) | (b[:, 1] != 0)] for b in res.buffers])
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))
