"""Property tests of the reference's own DPU join kernels (compiled from the
reference tree and run on the host, oracle/dpu_ref.py) against the oracle:
hypothesis draws small relations with repeated keys, (0, 0) padding, one-key
domains and empty inputs, and every kernel's result must equal the oracle's.
Skipped where the runners were not built or hypothesis is missing."""
import numpy as np
import pytest

import dpu_ref

pytestmark = pytest.mark.skipif(not dpu_ref.available(), reason="reference DPU kernels not built here")
hyp = pytest.importorskip("hypothesis")
st = hyp.strategies


def _random_relations(seed, n_r, n_s, domain, zero_every):
    """Small relations for property tests: keys from 1..domain (repeats in R
    and S), R payloads = R index (so a pair names its R tuple), some (0, 0)
    padding as the reference's packets carry it, S keys partly outside R's
    domain and all below 2^31."""
    rng = np.random.default_rng(seed)
    R = np.stack([rng.integers(1, domain + 1, n_r), np.arange(n_r)], 1).astype(np.uint32).reshape(n_r, 2)
    s_hi = min(2 * domain + 2, 1 << 31)  # keys stay below 2^31, as the reference's kernels require
    S = np.stack([rng.integers(1, s_hi, n_s), np.arange(n_s)], 1).astype(np.uint32).reshape(n_s, 2)
    if zero_every:
        R[::zero_every] = 0
        S[::zero_every] = 0
    return R, S


def _check_first_match_join(oracle, R, S, got):
    """Pairs of a first-match join with repeated R keys: the same S tuples as
    the oracle's, each joined with an R tuple of its key."""
    want = oracle.simple_join(R, S)
    assert got.shape == want.shape
    assert np.array_equal(np.sort(got[:, 1]), np.sort(want[:, 1]))
    if got.shape[0]:
        assert np.array_equal(R[got[:, 0], 0], S[got[:, 1], 0])


@hyp.settings(max_examples=20, deadline=None)
@hyp.given(seed=st.integers(0, 2**32 - 1), n_r=st.integers(0, 1900), n_s=st.integers(0, 4000),
           domain=st.sampled_from([1, 7, 300, 5000, 2**31 - 1]), zero_every=st.sampled_from([0, 1, 3, 97]))
def test_property_hash_kernels(oracle, seed, n_r, n_s, domain, zero_every):
    """Local partitioning, build and probe on one DPU (the reference's
    kernels) against the oracle, over sizes 0 ... 1900 x 0 ... 4000, key
    domains from one key to 2^31, and padding from none to all."""
    R, S = _random_relations(seed, n_r, n_s, domain, zero_every)
    rg, ro, L = dpu_ref.local_partition(R)
    sg, so, _ = dpu_ref.local_partition(S, partitions=L)
    if int(np.diff(ro).max(initial=0)) > dpu_ref.TABLE_BYTES // 8:
        return  # a partition beyond the kernel's table (it would never finish): not a case it runs
    _check_first_match_join(oracle, R, S, dpu_ref.hash_join(rg, ro, sg, so))


@hyp.settings(max_examples=20, deadline=None)
@hyp.given(seed=st.integers(0, 2**32 - 1), n_r=st.integers(0, 3000), n_s=st.integers(0, 6000),
           domain=st.sampled_from([1, 7, 300, 5000, 2**31 - 1]), zero_every=st.sampled_from([0, 1, 3, 97]))
def test_property_nphj_kernels(oracle, seed, n_r, n_s, domain, zero_every):
    """The non-partitioned build and probe against the oracle on the same
    random relations."""
    R, S = _random_relations(seed, n_r, n_s, domain, zero_every)
    _check_first_match_join(oracle, R, S, dpu_ref.nphj(R, S)[0])


@hyp.settings(max_examples=15, deadline=None)
@hyp.given(seed=st.integers(0, 2**32 - 1), n_r=st.integers(0, 700), n_s=st.integers(0, 1500),
           domain=st.sampled_from([7, 300, 5000]), zero_every=st.sampled_from([0, 3, 97]))
def test_property_nested_loop_kernel(oracle, seed, n_r, n_s, domain, zero_every):
    """The nested-loop kernel's rewritten S against the oracle's
    keep-unmatched join, row for row, with R payloads above every key (so its
    second rewrite cannot occur) and repeated R keys (the first R tuple in R
    order wins). The kernel compares key 0 like any key, so a (0, 0) padding
    tuple of S "joins" R's padding and stays (0, 0); the oracle emits no row
    for padding."""
    R, S = _random_relations(seed, n_r, n_s, domain, zero_every)
    live = R[:, 0] != 0
    R[live, 1] += np.uint32(1 << 31)
    got = dpu_ref.nested_loop(R, S)
    pad = S[:, 0] == 0
    assert not got[pad].any()
    assert np.array_equal(got[~pad], oracle.simple_join(R, S, keep_unmatched=True))


@hyp.settings(max_examples=20, deadline=None)
@hyp.given(seed=st.integers(0, 2**32 - 1), n=st.integers(0, 6000), log_p=st.integers(0, 11),
           log_g=st.integers(0, 4), zero_every=st.sampled_from([0, 1, 5]))
def test_property_count_kernel(oracle, seed, n, log_p, log_g, zero_every):
    """The global partition count against the oracle for any power-of-two
    fan-out up to 2048 and, when the rank sets divide it, the rank-set split."""
    P, G = 1 << log_p, 1 << log_g
    T, _ = _random_relations(seed, n, 0, 2**31 - 1, zero_every)
    type_ = 1 if G > 1 and P % (64 * G) == 0 else 0
    rps = P // 64 // G if type_ else 1
    hist, _ = dpu_ref.partition_count(T, P, type_, G if type_ else 1, rps)
    assert np.array_equal(hist, oracle.partition_count(T, P, type_, G if type_ else 1, rps))


@hyp.settings(max_examples=15, deadline=None)
@hyp.given(seed=st.integers(0, 2**32 - 1), n=st.integers(0, 5000), log_ranks=st.integers(0, 3),
           log_g=st.integers(0, 3), dpu_id=st.integers(0, 63), log_packet=st.integers(3, 7),
           bank_set=st.sampled_from([1, 8, 16, 32, 64]), zero_every=st.sampled_from([0, 2, 97]))
def test_property_packet_scatters(oracle, seed, n, log_ranks, log_g, dpu_id, log_packet, bank_set, zero_every):
    """The plain and chip-wise packet scatters against the oracle's
    destinations for random blocks, rank counts, rank sets, source DPUs,
    packet sizes and bank sets."""
    ranks = 1 << log_ranks
    G = 1 << min(log_g, log_ranks)
    if bank_set > 1 and ranks // G * 64 < bank_set:
        return
    T, _ = _random_relations(seed, n, 0, 2**31 - 1, zero_every)
    groups = dpu_ref.packet_scatter(T, ranks, G, dpu_id, 1 << log_packet, bank_set=bank_set)
    if bank_set > 1:
        dest = oracle.chipwise_partition_dest(T, ranks, G, bank_set)
    else:
        dest = oracle.partition_dest(T, 64 * ranks, 0 if G == 1 else 1, G, ranks // G)
    for d, g in enumerate(groups):
        assert np.array_equal(oracle.sort_pairs(g), oracle.sort_pairs(T[dest == d]))
