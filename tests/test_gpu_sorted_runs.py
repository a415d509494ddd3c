"""The sort-merge join sorts every R partition once, in runs that fit a CTA's
shared memory; a partition larger than that (many repeats of one key) is
searched run by run in global memory, by the sort-merge and the nested-loop
joins alike, instead of failing. Exact against the oracle where R keys are
unique; count and validity where they repeat (which repeated R tuple a probe
returns is unspecified, as in the reference)."""
import numpy as np
import pytest

from test_gpu_parity import run_instance, same_multiset

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alg", [2, 3])
def test_r_partition_beyond_shared_memory(spj, oracle, alg):
    rng = np.random.default_rng(12)
    n_u = 1 << 15
    keys = np.concatenate([rng.permutation(np.arange(1, n_u + 1)), np.full(60000, 9)])  # key 9: 60001 times
    R = np.stack([keys, np.arange(keys.size)], 1).astype(np.uint32)
    sk = rng.integers(1, 2 * n_u, 1 << 19)  # half of them miss R: kept unchanged by SMJ / NL
    sk[rng.random(sk.size) < 0.1] = 9
    S = np.stack([sk, np.arange(sk.size)], 1).astype(np.uint32)
    res, logs = run_instance(spj, R, S, join_alg=alg, heavy_sample=-1)
    out = res.pairs()
    assert out.shape[0] == S.shape[0]
    hit = S[:, 0] <= n_u
    by_s = np.empty_like(out)
    by_s[out[:, 1]] = out
    assert np.array_equal(np.sort(out[:, 1]), np.arange(S.shape[0], dtype=np.uint32))
    assert np.array_equal(by_s[~hit, 0], S[~hit, 0])            # unmatched: (S.key, S.pay)
    assert np.array_equal(R[by_s[hit, 0], 0], S[hit, 0])       # matched: an R row of the same key


@pytest.mark.parametrize("zipf", [0.0, 1.5])
def test_sort_merge_sorted_once_exact(spj, oracle, zipf):
    R, S, expect = spj.generate_host(1 << 18, 1 << 21, zipf, seed=41)
    for layout in ((1, 1, 1, 0), (4, 4, 1, 1)):
        ranks, rsets, bset, mode = layout
        res, _ = run_instance(spj, R, S, ranks=ranks, rank_sets=rsets, bank_set=bset, skew_mode=mode, join_alg=2)
        out = res.pairs()
        assert oracle.checksum(out) == expect
        assert same_multiset(oracle, out, oracle.simple_join(R, S, keep_unmatched=True))


def test_sort_merge_bucket_sort_fallback(spj, oracle):
    """A run's bucket sort spreads its keys over [min, max]; one key near 2^32 in
    a partition of small keys puts nearly all of them in the first bucket, which
    makes that run fall back to the merge sort. Runs with and without the
    fallback give the oracle's keep-unmatched join exactly."""
    rng = np.random.default_rng(29)
    n_small = 1 << 18
    keys = rng.permutation(np.arange(1, n_small + 1)).astype(np.uint64)
    far = (np.uint64(2**32) - np.arange(1, 4097, dtype=np.uint64))  # one far key in most partitions
    R = np.stack([np.concatenate([keys, far]), np.arange(n_small + far.size)], 1).astype(np.uint32)
    sk = np.concatenate([rng.integers(1, 2 * n_small, 1 << 20), far[rng.integers(0, far.size, 1 << 14)]])
    S = np.stack([sk, np.arange(sk.size)], 1).astype(np.uint32)
    res, _ = run_instance(spj, R, S, join_alg=2, heavy_sample=-1)
    assert same_multiset(oracle, res.pairs(), oracle.simple_join(R, S, keep_unmatched=True))
