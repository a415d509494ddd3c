"""CPU tests of the oracle: pinned against the reference's own hash functions
(compiled from its source into the golden vectors) and the known answers of the
reference's synthetic driver, then checked for internal consistency."""
import json
import os

import numpy as np
import pytest

from conftest import main_cc_tables

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_hashes_match_reference_hash_c(oracle):
    g = load("hash_vectors.json")
    got = oracle.hashes(g["keys"])
    for col, name in enumerate(["glb_partition_hash", "local_partition_hash", "join_hash", "join_hash2"]):
        assert got[:, col].tolist() == g[name], name
    tab = oracle.lib().orc_crc_table()
    assert [tab[i] for i in range(256)] == g["crctab"]


def test_vectorised_partition_hash_matches(oracle):
    g = load("hash_vectors.json")
    assert oracle.glb_partition_hash_np(g["keys"]).tolist() == g["glb_partition_hash"]


@pytest.mark.parametrize("case", load("kat_main_cc.json")["cases"], ids=lambda c: f"N{c['N']}x{c['ratio']}")
def test_kat_main_cc_simple_and_refpipe(oracle, case):
    R, S = main_cc_tables(case["N"], case["ratio"])
    for out in (oracle.simple_join(R, S),
                oracle.refpipe_join(R, S, ranks=1),
                oracle.refpipe_join(R, S, ranks=4, rank_sets=2),
                oracle.refpipe_join(R, S, ranks=2, rank_sets=1, bank_set=16)):
        assert out.shape[0] == case["n_pairs"]
        assert oracle.checksum(out) == case["checksum"]
        srt = oracle.sort_pairs(out)
        assert srt[:len(case["first_sorted"])].tolist() == case["first_sorted"]


@pytest.mark.parametrize("alg", [0, 2, 3])
@pytest.mark.parametrize("layout", [(1, 1, 1), (2, 2, 1), (4, 1, 8), (2, 2, 32), (1, 1, 64)])
def test_refpipe_equals_simple_on_fk(oracle, spj, alg, layout):
    ranks, rsets, bset = layout
    for zipf in (0.0, 1.0, 1.5):
        R, S, expect = spj.generate_host(5000, 20000, zipf, seed=7 + int(zipf * 10))
        a = oracle.sort_pairs(oracle.refpipe_join(R, S, ranks, rsets, bset, alg))
        b = oracle.sort_pairs(oracle.simple_join(R, S))
        assert np.array_equal(a, b)
        assert oracle.checksum(a) == expect


def test_refpipe_semantics_non_fk(oracle):
    rng = np.random.default_rng(3)
    R = np.stack([rng.permutation(np.arange(1, 3001)), np.arange(3000)], 1).astype(np.uint32)
    S = np.stack([rng.integers(0, 6000, 9000), np.arange(9000)], 1).astype(np.uint32)  # half miss, some key 0
    inner = oracle.sort_pairs(oracle.simple_join(R, S))
    keep = oracle.sort_pairs(oracle.simple_join(R, S, keep_unmatched=True))
    assert np.array_equal(oracle.sort_pairs(oracle.refpipe_join(R, S, alg=0)), inner)
    for alg in (2, 3):
        assert np.array_equal(oracle.sort_pairs(oracle.refpipe_join(R, S, alg=alg)), keep)
    valid = int((S[:, 0] != 0).sum())
    assert keep.shape[0] == valid
    assert inner.shape[0] == int(((S[:, 0] >= 1) & (S[:, 0] <= 3000)).sum())


def test_refpipe_duplicate_r_keys_first_in_r_order(oracle):
    R = np.array([[5, 100], [7, 200], [5, 101], [9, 300], [5, 102]], dtype=np.uint32)
    S = np.array([[5, 1], [9, 2], [8, 3], [5, 4], [0, 5]], dtype=np.uint32)
    want = [[100, 1], [100, 4], [300, 2]]
    for alg in (0, 2, 3):
        got = oracle.sort_pairs(oracle.refpipe_join(R, S, alg=alg))
        exp = want if alg == 0 else sorted(want + [[8, 3]])
        assert got.tolist() == exp


def test_key_zero_never_joins(oracle):
    R = np.array([[0, 1], [0, 2], [3, 4]], dtype=np.uint32)
    S = np.array([[0, 10], [3, 11], [0, 12]], dtype=np.uint32)
    for out in (oracle.simple_join(R, S), oracle.refpipe_join(R, S)):
        assert out.tolist() == [[4, 11]]


def test_empty_and_single(oracle):
    z = np.zeros((0, 2), dtype=np.uint32)
    one = np.array([[42, 7]], dtype=np.uint32)
    assert oracle.refpipe_join(z, one).shape[0] == 0
    assert oracle.refpipe_join(one, z).shape[0] == 0
    assert oracle.refpipe_join(one, one).tolist() == [[7, 7]]
    assert oracle.refpipe_join(z, one, alg=3).tolist() == [[42, 7]]


def test_table_full_is_reported(oracle):
    # 5000 copies of one key land in one local partition (> 4096 slots); the
    # reference's build would spin forever (a2a_srj_build.c:225-281)
    R = np.stack([np.full(5000, 77), np.arange(5000)], 1).astype(np.uint32)
    S = np.array([[77, 1]], dtype=np.uint32)
    with pytest.raises(RuntimeError, match="4096"):
        oracle.refpipe_join(R, S, ranks=1)


def test_partition_count_restatement(oracle, spj):
    R, S, _ = spj.generate_host(4096, 8192, 0.0, seed=11)
    for P in (64, 256, 4096):
        h = oracle.partition_count(R, P)
        ref = np.bincount(oracle.glb_partition_hash_np(R[:, 0]) & (P - 1), minlength=P)
        assert np.array_equal(h, ref)
    # S with 4 rank sets: the set comes from the index inside each 256-tuple block
    h = oracle.partition_count(S, 256, type_=1, rank_sets=4, ranks_per_set=1)
    j = np.arange(S.shape[0]) & 255
    ids = (oracle.glb_partition_hash_np(S[:, 0]) & 63) + (j & 3) * 64
    assert np.array_equal(h, np.bincount(ids, minlength=256))


@pytest.mark.parametrize("layout", [(1, 1, 1), (4, 2, 1), (2, 1, 8), (2, 2, 16)])
def test_refpipe_replication_sizes(oracle, spj, layout):
    ranks, rsets, bset = layout
    R, S, _ = spj.generate_host(3000, 9000, 1.0, seed=5)
    rs, ss = oracle.refpipe_dpu_sizes(R, S, ranks, rsets, bset)
    assert rs.sum() == 3000 * rsets * bset   # every R tuple on every replica of its partition
    assert ss.sum() == 9000                  # every S tuple on exactly one replica


@pytest.mark.parametrize("n_r,n_s,zipf,seed", [(1000, 5000, 0.0, 3), (1 << 16, 1 << 18, 1.0, 2024),
                                               (12345, 99999, 1.5, 7), (1 << 20, 1 << 21, 0.0, 0x5EED5EED)])
def test_oracle_generator_equals_product_host_generator(oracle, spj, n_r, n_s, zipf, seed):
    """The oracle's restated generator (used by the CPU arms of the benchmark,
    which load no product library) gives the product generator's bytes and
    expected checksum."""
    R, S, e = oracle.generate(n_r, n_s, zipf, seed=seed)
    R2, S2, e2 = spj.generate_host(n_r, n_s, zipf, seed=seed)
    assert np.array_equal(R, R2) and np.array_equal(S, S2) and e == e2
    assert oracle.checksum(oracle.simple_join_mt(R, S)) == e


def test_threaded_join_and_sort_equal_single_threaded(oracle):
    rng = np.random.default_rng(11)
    # repeated R keys (the first in R order wins), key-0 padding, unmatched S keys
    R = np.stack([rng.integers(0, 3000, 20000), rng.integers(0, 2**32, 20000)], axis=1).astype(np.uint32)
    S = np.stack([rng.integers(0, 4000, 90000), np.arange(90000)], axis=1).astype(np.uint32)
    for keep in (False, True):
        a = oracle.simple_join(R, S, keep_unmatched=keep)
        for t in (1, 3, 8):
            assert np.array_equal(a, oracle.simple_join_mt(R, S, keep_unmatched=keep, nthreads=t))
    for t in (1, 5, 16):
        assert np.array_equal(oracle.sort_pairs(S), oracle.sort_pairs_mt(S, nthreads=t))


def test_select_restates_the_reference_predicates(oracle):
    rng = np.random.default_rng(21)
    T = np.stack([rng.integers(0, 1000, 5000), rng.integers(0, 2**32, 5000)], 1).astype(np.uint32)
    cmp = {0: lambda v, a, b: v == a, 1: lambda v, a, b: v <= a, 2: lambda v, a, b: v >= a,
           3: lambda v, a, b: v < a, 4: lambda v, a, b: v > a, 5: lambda v, a, b: a <= v <= b}
    for field in (1, 2):
        for op in range(6):
            lo = 500 if field == 1 else 2**31
            hi = 700 if field == 1 else 2**32 - 5
            want = [tuple(t) for t in T.tolist() if cmp[op](t[field - 1], lo, hi)]
            got = oracle.select(T, field, op, lo, hi)
            assert [tuple(t) for t in got.tolist()] == want, (field, op)
    assert np.array_equal(oracle.select(T, 0), T)
