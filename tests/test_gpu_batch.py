"""GPU tests of the batched form: many joins of uneven sizes, R:S ratios and
skew in one launch sequence, each join's output checked against its exact
answer (the generator's checksum) and, for small joins, the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_batch_inputs(spj, specs, seed0=100):
    import torch
    R, S, exp = [], [], []
    for i, (n_r, n_s, z) in enumerate(specs):
        dR = torch.empty((max(n_r, 1), 2), dtype=torch.int32, device="cuda")
        dS = torch.empty((max(n_s, 1), 2), dtype=torch.int32, device="cuda")
        e = torch.zeros(1, dtype=torch.int64, device="cuda")
        spj.check(spj.lib().spj_generate_device(seed0 + i, n_r, n_s, z, dR.data_ptr(), dS.data_ptr(),
                                                e.data_ptr(), None))
        R.append(dR)
        S.append(dS)
        exp.append(e)
    torch.cuda.synchronize()
    return R, S, [int(e.item()) for e in exp]


def run_batch(spj, specs, design, R, S, graph=False, repeats=2):
    import torch
    J = len(specs)
    b = spj.Batch([x[0] for x in specs], [x[1] for x in specs], design)
    outs = [torch.empty((b.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(J)]
    n_out = torch.zeros(J, dtype=torch.int64, device="cuda")
    b.bind([t.data_ptr() for t in R], [t.data_ptr() for t in S], [o.data_ptr() for o in outs], n_out.data_ptr())
    results = []
    if graph:
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            b.execute(s.cuda_stream)  # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            b.execute(torch.cuda.current_stream().cuda_stream)
        for _ in range(repeats):
            n_out.zero_()
            g.replay()
            torch.cuda.synchronize()
            results.append([outs[j][:int(n_out[j].item())].cpu().numpy().view(np.uint32) for j in range(J)])
    else:
        for _ in range(repeats):
            n_out.zero_()
            b.execute(0)
            torch.cuda.synchronize()
            results.append([outs[j][:int(n_out[j].item())].cpu().numpy().view(np.uint32) for j in range(J)])
    stats = [b.stats(j) for j in range(J)]
    b.close()
    return results, stats


SPECS = [(1 << 12, 1 << 12, 0.0), (5000, 40000, 1.2), (1 << 16, 1 << 18, 1.5), (3, 7, 0.0), (1 << 20, 1 << 21, 0.7),
         (123457, 493828, 1.0), (1 << 14, 1 << 17, 0.3), (1 << 18, 1 << 18, 1.5), (0, 100, 0.0), (77, 0, 0.0)]


@pytest.mark.parametrize("alg", ["phj", "nphj", "smj", "nl"])
def test_batch_each_join_exact(spj, oracle, alg):
    specs = [s for s in SPECS if s[0] > 0]  # the generator needs |R| >= 1
    R, S, exp = make_batch_inputs(spj, specs)
    results, stats = run_batch(spj, specs, spj.make_design(rank_num=1, join_alg=alg), R, S)
    for rep in results:
        for j, (n_r, n_s, z) in enumerate(specs):
            out = rep[j]
            assert out.shape[0] == n_s, (alg, j)
            assert oracle.checksum(out) == exp[j] & (2**64 - 1), (alg, j)
    for j, (n_r, n_s, z) in enumerate(specs):
        if n_r * n_s and n_s <= 1 << 18:
            Rh = R[j].cpu().numpy().view(np.uint32)[:n_r]
            Sh = S[j].cpu().numpy().view(np.uint32)[:n_s]
            ref = oracle.sort_pairs(oracle.simple_join(Rh, Sh))
            assert np.array_equal(oracle.sort_pairs(results[0][j]), ref), (alg, j)


def test_batch_with_empty_relations(spj, oracle):
    import torch
    specs = [(0, 100), (77, 0), (1000, 3000)]
    rng = np.random.default_rng(1)
    host = []
    for n_r, n_s in specs:
        Rh = np.stack([rng.permutation(np.arange(1, n_r + 1)), np.arange(n_r)], 1).astype(np.uint32).reshape(n_r, 2)
        Sh = np.stack([rng.integers(1, n_r + 2, n_s), np.arange(n_s)], 1).astype(np.uint32).reshape(n_s, 2)
        host.append((Rh, Sh))
    R = [torch.from_numpy(np.vstack([h[0], np.zeros((1, 2), np.uint32)]).view(np.int32)).cuda() for h in host]
    S = [torch.from_numpy(np.vstack([h[1], np.zeros((1, 2), np.uint32)]).view(np.int32)).cuda() for h in host]
    results, _ = run_batch(spj, [(a, b, 0.0) for a, b in specs], spj.make_design(rank_num=1), R, S, repeats=1)
    for j, (Rh, Sh) in enumerate(host):
        assert np.array_equal(oracle.sort_pairs(results[0][j]), oracle.sort_pairs(oracle.simple_join(Rh, Sh)))


def test_batch_cuda_graph_replay(spj, oracle):
    specs = [s for s in SPECS if s[0] > 0]
    R, S, exp = make_batch_inputs(spj, specs, seed0=500)
    results, _ = run_batch(spj, specs, spj.make_design(rank_num=1), R, S, graph=True, repeats=3)
    for rep in results:
        for j, (n_r, n_s, z) in enumerate(specs):
            assert rep[j].shape[0] == n_s
            assert oracle.checksum(rep[j]) == exp[j] & (2**64 - 1)


def test_batch_matches_plain_plans(spj, oracle):
    """The batch gives every join the same pair multiset as a plain plan of that join."""
    import torch
    specs = [(1 << 15, 1 << 17, 1.1), (20000, 20000, 0.0), (1 << 17, 1 << 19, 1.4)]
    R, S, exp = make_batch_inputs(spj, specs, seed0=900)
    results, _ = run_batch(spj, specs, spj.make_design(rank_num=1), R, S, repeats=1)
    for j, (n_r, n_s, z) in enumerate(specs):
        plan = spj.Plan(n_r, n_s, spj.make_design(rank_num=1))
        out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
        n = torch.zeros(1, dtype=torch.int64, device="cuda")
        plan.execute(R[j].data_ptr(), S[j].data_ptr(), out.data_ptr(), n.data_ptr(), 0)
        torch.cuda.synchronize()
        plain = out[:int(n.item())].cpu().numpy().view(np.uint32)
        plan.close()
        assert np.array_equal(oracle.sort_pairs(plain), oracle.sort_pairs(results[0][j]))


def test_autotuned_batch_stays_exact(spj, oracle):
    table = spj.autotune([(12, 1), (14, 0)], zipf=1.0, reps=1, batch_tuples=1 << 20, max_joins=8,
                         candidates=[(0, 0, 0), (1, 0, 0), (-1, 0, 32768)])
    assert len(table) == 2 and all(e["ms"] > 0 for e in table)
    spj.set_tuning(table)
    try:
        specs = [(1 << 12, 1 << 13, 1.0), (1 << 14, 1 << 14, 0.5), (5000, 9000, 1.2)] * 2
        R, S, exp = make_batch_inputs(spj, specs, seed0=900)
        results, _ = run_batch(spj, specs, spj.make_design(rank_num=1), R, S, repeats=1)
        for j, (n_r, n_s, _) in enumerate(specs):
            assert results[0][j].shape == (n_s, 2)
            assert oracle.checksum(results[0][j]) == exp[j] & (2**64 - 1)
    finally:
        spj.set_tuning([])


@pytest.mark.parametrize("design_alg,table", [
    (0, [{"log2_r": 12, "log2_ratio": 1, "join_alg": 2}, {"log2_r": 16, "log2_ratio": 2, "join_alg": 1}]),
    (2, [{"log2_r": 12, "log2_ratio": 1, "join_alg": 4}, {"log2_r": 16, "log2_ratio": 2, "join_alg": 3}]),
    (0, [{"log2_r": 12, "log2_ratio": 1, "join_alg": 3}]),  # another output semantics: ignored
])
def test_batch_mixes_local_join_algorithms(spj, oracle, design_alg, table):
    """A tuning table can give size classes their own local-join algorithm (among
    those with the design's output semantics): one batch then runs the hash and
    non-partitioned hash joins, or sort-merge and nested loop, side by side, each
    over its own range of work units; every join equals the oracle."""
    rng = np.random.default_rng(77)
    specs = [(1 << 12, 1 << 13, 1.0), (1 << 16, 1 << 18, 1.2), (70000, 150000, 0.0), (1 << 12, 9000, 0.5)]
    data = []
    for n_r, n_s, z in specs:
        R, S, _ = spj.generate_host(n_r, n_s, z, seed=int(rng.integers(1 << 30)))
        S[::7, 0] = 0xFFFFFFF0  # unmatched S tuples: dropped by the hash joins, kept by SMJ / NL
        data.append((R, S))
    import torch
    R = [torch.from_numpy(r.view(np.int32)).cuda() for r, _ in data]
    S = [torch.from_numpy(x.view(np.int32)).cuda() for _, x in data]
    spj.set_tuning(table)
    try:
        results, _ = run_batch(spj, specs, spj.make_design(rank_num=1, join_alg=design_alg), R, S)
    finally:
        spj.set_tuning([])
    for rep in results:
        for j, (r, x) in enumerate(data):
            want = oracle.simple_join(r, x, keep_unmatched=design_alg in (2, 3))
            assert np.array_equal(oracle.sort_pairs(rep[j]), oracle.sort_pairs(want)), j
