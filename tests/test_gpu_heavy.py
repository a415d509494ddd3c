"""GPU parity of the heavy-key path: S keys that a sample of S shows to be
frequent are joined on the fly in the first scatter pass (their R payloads found
by the count pass over R) instead of being partitioned. The output must equal
the oracle's join exactly with the path on or off, for every local join, for
unmatched heavy keys (dropped by the hash join, kept by sort-merge and nested
loop, which rewrite S in place), in batches and in the sliced JoinInstance path
that reuses R's partitions."""
import numpy as np
import pytest

from test_gpu_parity import run_instance as _run_instance, same_multiset

pytestmark = pytest.mark.gpu


def run_instance(spj, R, S, **kw):
    """The partitioned joins (the planner runs a small R alone without
    partitions, where no heavy keys are sampled): an explicit fan-out for the
    hash join."""
    if kw.get("join_alg", 0) == 0:
        kw.setdefault("radix_bits", 11)
    return _run_instance(spj, R, S, **kw)


@pytest.mark.parametrize("alg", [0, 2, 3])
def test_heavy_keys_zipf_1_5_exact_and_counted(spj, oracle, alg):
    R, S, expect = spj.generate_host(1 << 18, 1 << 20, 1.5, seed=77)
    res, logs = run_instance(spj, R, S, join_alg=alg, heavy_sample=1 << 14)
    out = res.pairs()
    assert out.shape[0] == S.shape[0] and oracle.checksum(out) == expect
    assert same_multiset(oracle, out, oracle.simple_join(R, S))
    # Zipf 1.5 over 2^18 keys: the top 256 keys hold about 95% of S
    assert 0 < logs["heavy_keys"] <= 256
    assert logs["heavy_tuples"] > 0.8 * S.shape[0]


def test_heavy_path_off_gives_the_same_pairs(spj, oracle):
    R, S, expect = spj.generate_host(1 << 17, 1 << 20, 1.0, seed=78)
    on, lon = run_instance(spj, R, S, heavy_sample=1 << 16)
    off, loff = run_instance(spj, R, S, heavy_sample=-1)
    assert loff["heavy_keys"] == 0 and loff["heavy_tuples"] == 0 and lon["heavy_keys"] > 0
    assert same_multiset(oracle, on.pairs(), off.pairs())
    assert oracle.checksum(off.pairs()) == expect


@pytest.mark.parametrize("alg", [0, 2, 3])
def test_heavy_keys_without_r_match(spj, oracle, alg):
    """Two hot S keys, one absent from R: the hash join drops its tuples, the
    sort-merge and nested-loop joins keep them unchanged."""
    rng = np.random.default_rng(9)
    n_r, n_s = 1 << 16, 1 << 20
    R = np.stack([rng.permutation(np.arange(1, n_r + 1)), rng.integers(0, 2**32, n_r)], 1).astype(np.uint32)
    keys = rng.integers(1, 2 * n_r, n_s)          # half of the cold keys miss R too
    u = rng.random(n_s)
    keys[u < 0.35] = 7                            # in R
    keys[(u >= 0.35) & (u < 0.6)] = 3 * n_r + 5   # not in R
    S = np.stack([keys, np.arange(n_s)], 1).astype(np.uint32)
    res, logs = run_instance(spj, R, S, join_alg=alg, heavy_sample=1 << 16)
    want = oracle.simple_join(R, S, keep_unmatched=alg in (2, 3))
    assert same_multiset(oracle, res.pairs(), want)
    assert logs["heavy_keys"] >= 2


def test_heavy_key_repeated_in_r(spj, oracle):
    """A hot key held by several R tuples: each S tuple still gets exactly one
    pair, with the payload of one of those R tuples."""
    rng = np.random.default_rng(10)
    n_r, n_s = 1 << 16, 1 << 20
    keys_r = np.concatenate([rng.permutation(np.arange(1, n_r + 1)), np.full(5, 11)])  # key 11 six times
    R = np.stack([keys_r, np.arange(n_r + 5)], 1).astype(np.uint32)
    keys = rng.integers(1, n_r + 1, n_s)
    keys[rng.random(n_s) < 0.5] = 11
    S = np.stack([keys, np.arange(n_s)], 1).astype(np.uint32)
    res, logs = run_instance(spj, R, S, heavy_sample=1 << 16)
    out = res.pairs()
    assert logs["heavy_keys"] >= 1
    assert out.shape[0] == n_s
    assert np.array_equal(np.sort(out[:, 1]), np.arange(n_s, dtype=np.uint32))
    assert np.array_equal(R[out[:, 0], 0], S[out[:, 1], 0])


def test_automatic_mode_keeps_heavy_keys_only_under_strong_skew(spj):
    """The planner's sample keeps its heavy keys only when they hold most of S:
    on for Zipf 1.5, off for Zipf 1.0 (where a filter lookup per tuple would
    cost more than the partitioning it saves) and for uniform keys."""
    for zipf, on in ((1.5, True), (1.0, False), (0.0, False)):
        # |R| = 2^23: above the size the planner joins without partitions
        R, S, expect = spj.generate_host(1 << 23, 1 << 24, zipf, seed=80)
        res, logs = _run_instance(spj, R, S)
        assert (logs["heavy_keys"] > 0) == on, zipf


def test_heavy_keys_in_a_batch(spj, oracle):
    import torch
    specs = [(1 << 16, 1 << 20, 1.5), (1 << 12, 1 << 20, 1.2), (1 << 18, 1 << 18, 1.0), (5000, 1 << 21, 0.0)]
    data = [spj.generate_host(a, b, z, seed=90 + i) for i, (a, b, z) in enumerate(specs)]
    batch = spj.Batch([a for a, _, _ in specs], [b for _, b, _ in specs],
                      spj.make_design(rank_num=1, heavy_sample=1 << 16))
    dR = [torch.from_numpy(R.view(np.int32)).cuda() for R, _, _ in data]
    dS = [torch.from_numpy(S.view(np.int32)).cuda() for _, S, _ in data]
    outs = [torch.empty((batch.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(len(specs))]
    n_out = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    batch.bind([t.data_ptr() for t in dR], [t.data_ptr() for t in dS], [o.data_ptr() for o in outs],
               n_out.data_ptr())
    for _ in range(2):
        batch.execute(0)
        torch.cuda.synchronize()
        for j, (R, S, expect) in enumerate(data):
            k = int(n_out[j].item())
            got = outs[j][:k].cpu().numpy().view(np.uint32)
            assert k == S.shape[0] and oracle.checksum(got) == expect
            assert same_multiset(oracle, got, oracle.simple_join(R, S))
    assert batch.stats(0)["heavy_keys"] > 0
    batch.close()


def test_heavy_keys_with_host_slices(spj, oracle):
    """|S| >= 2^24 in host memory: S is joined in slices that reuse R's
    partitions and the heavy table of the first slice."""
    R, S, expect = spj.generate_host(1 << 20, 1 << 25, 1.5, seed=95)
    res, logs = run_instance(spj, R, S, heavy_sample=1 << 14)
    out = res.pairs()
    assert out.shape[0] == S.shape[0] and oracle.checksum(out) == expect
    assert logs["heavy_keys"] > 0
