"""spj_join_noalloc: the join for callers that cannot allocate device memory
while they run it (a database engine whose pool allocator owns the whole GPU, a
loop that must not stall on cudaMalloc/cudaFree). Its output must equal that
of the regular entry point, spj_plan_execute, bit for bit (the pair multiset,
compared after a canonical sort), on consecutive calls that reuse its fixed
scratch region. This file is collected last on purpose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _plan_join(spj, dR, dS, n_r, n_s):
    """The regular entry point (scratch allocated by spj_plan_create)."""
    import torch
    plan = spj.Plan(n_r, n_s, spj.make_design(rank_num=1))
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n.data_ptr(), 0)
    torch.cuda.synchronize()
    plan.close()
    k = int(n.item())
    return out[:k].cpu().numpy().view(np.uint32)


def _noalloc_join(spj, dR, dS, n_r, n_s):
    import torch
    cap = n_s + (1 << 21)
    out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_join_noalloc(dR.data_ptr(), n_r, dS.data_ptr(), n_s, out.data_ptr(), cap,
                                         n.data_ptr(), None))
    torch.cuda.synchronize()
    k = int(n.item())
    assert k >= 0, f"capacity error reported: {k}"
    return out[:k].cpu().numpy().view(np.uint32)


def test_noalloc_matches_plan_execute_on_consecutive_calls(spj, oracle):
    # two calls in a row: the second one finds the first one's data in the region
    cases = [(1 << 20, 1 << 21, 1.0, 11), (40000, 300001, 0.0, 12), (1 << 20, 1 << 21, 1.5, 13)]
    for n_r, n_s, zipf, seed in cases:
        R, S, expect = spj.generate_host(n_r, n_s, zipf, seed=seed)
        dR, dS = _device(R), _device(S)
        want = _plan_join(spj, dR, dS, n_r, n_s)
        got = _noalloc_join(spj, dR, dS, n_r, n_s)
        assert got.shape == want.shape == (n_s, 2)
        assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))
        assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))
        assert oracle.checksum(got) == expect


def test_noalloc_non_fk_against_oracle(spj, oracle):
    """S keys absent from R, padding (key 0) in both relations, repeated S keys:
    the pairs equal the oracle's independent join."""
    rng = np.random.default_rng(23)
    n_r, n_s = 300000, (1 << 21) - 5
    R = np.stack([rng.permutation(np.arange(1, 2 * n_r + 1))[:n_r], rng.integers(0, 2**32, n_r)],
                 1).astype(np.uint32)
    R[::101, 0] = 0
    S = np.stack([rng.integers(0, 3 * n_r, n_s), np.arange(n_s)], 1).astype(np.uint32)
    got = _noalloc_join(spj, _device(R), _device(S), n_r, n_s)
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))


def test_noalloc_rejects_sizes_over_its_limit(spj):
    import torch
    d = torch.zeros((16, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(spj.SpjError, match="2\\^20"):
        spj.check(spj.lib().spj_join_noalloc(d.data_ptr(), (1 << 20) + 1, d.data_ptr(), 1, d.data_ptr(),
                                             1 << 22, n.data_ptr(), None))
    with pytest.raises(spj.SpjError, match="out_capacity"):
        spj.check(spj.lib().spj_join_noalloc(d.data_ptr(), 8, d.data_ptr(), 8, d.data_ptr(), 16,
                                             n.data_ptr(), None))


def _keys_in_one_partition(oracle, n, bits=8):
    """n distinct keys whose partition hash agrees in its low `bits` bits, so
    they share one partition of the entry point's one-pass plan (at most 2^8
    partitions)."""
    cand = np.arange(1, 1 << 24, dtype=np.uint32)
    keys = cand[(oracle.glb_partition_hash_np(cand) & ((1 << bits) - 1)) == 0]
    assert keys.size >= n
    return keys[:n]


def test_noalloc_reports_capacity_errors_and_recovers(spj, oracle):
    """An R whose keys all fall into one partition overflows that partition's
    shared-memory table: the count comes back negative with the table bit
    (error bit 1) set. The next call, on the same shared region, is exact again."""
    import torch
    keys = _keys_in_one_partition(oracle, 20000)
    R = np.stack([keys, np.arange(keys.size)], axis=1).astype(np.uint32)
    dR = _device(R)
    cap = R.shape[0] + (1 << 21)
    out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_join_noalloc(dR.data_ptr(), R.shape[0], dR.data_ptr(), R.shape[0], out.data_ptr(), cap,
                                         n.data_ptr(), None))
    torch.cuda.synchronize()
    k = int(n.item())
    assert k < 0 and ((-1 - k) & 1), f"expected the table-full status, got {k}"
    R2, S2, expect = spj.generate_host(1 << 20, 1 << 21, 1.0, seed=21)
    got = _noalloc_join(spj, _device(R2), _device(S2), 1 << 20, 1 << 21)
    assert got.shape[0] == 1 << 21 and oracle.checksum(got) == expect


def test_noalloc_call_leaves_free_device_memory_unchanged(spj):
    import torch
    R, S, _ = spj.generate_host(1 << 18, 1 << 20, 1.0, seed=31)
    dR, dS = _device(R), _device(S)
    cap = S.shape[0] + (1 << 21)
    out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    args = (dR.data_ptr(), R.shape[0], dS.data_ptr(), S.shape[0], out.data_ptr(), cap, n.data_ptr(), None)
    spj.check(spj.lib().spj_join_noalloc(*args))  # first call on the device: set-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        spj.check(spj.lib().spj_join_noalloc(*args))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(n.item()) == S.shape[0]


def test_noalloc_captured_in_a_cuda_graph(spj, oracle):
    """After one call (the per-device set-up), spj_join_noalloc is captured
    into a CUDA graph on a side stream in global capture mode, which fails any
    allocation or synchronisation inside the call. Two replays, each on new
    inputs copied into the same buffers, give those inputs' exact joins."""
    import torch
    n_r, n_s = 1 << 18, 1 << 20
    R0, S0, _ = spj.generate_host(n_r, n_s, 1.0, seed=41)
    dR, dS = _device(R0), _device(S0)
    cap = n_s + (1 << 21)
    out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    args = (dR.data_ptr(), n_r, dS.data_ptr(), n_s, out.data_ptr(), cap, n.data_ptr())
    spj.check(spj.lib().spj_join_noalloc(*args, None))
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side, capture_error_mode="global"):
        spj.check(spj.lib().spj_join_noalloc(*args, side.cuda_stream))
    for seed, zipf in ((42, 1.5), (43, 0.0)):
        R, S, expect = spj.generate_host(n_r, n_s, zipf, seed=seed)
        dR.copy_(_device(R))
        dS.copy_(_device(S))
        graph.replay()
        torch.cuda.synchronize()
        k = int(n.item())
        got = out[:k].cpu().numpy().view(np.uint32)
        assert k == n_s and oracle.checksum(got) == expect
        assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(oracle.simple_join(R, S)))
    del graph
