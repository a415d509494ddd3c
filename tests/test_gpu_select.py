"""GPU parity of the selections ahead of the join (the reference's TPC-H-style
predicates of src/dpu/include/select.h on a tuple's key or payload): spj_select
on its own, and the selections of a design applied inside the join's first
pass, against the oracle's restatement (select, then the independent join)."""
import numpy as np
import pytest

from test_gpu_parity import run_instance, same_multiset

pytestmark = pytest.mark.gpu

CASES = [(1, 0, 77, 0), (1, 1, 40000, 0), (1, 2, 40000, 0), (1, 3, 12345, 0), (1, 4, 99999, 0),
         (1, 5, 1000, 70000), (2, 5, 200000, 900000), (2, 3, 300000, 0), (0, 0, 0, 0)]


@pytest.mark.parametrize("field,op,lo,hi", CASES)
def test_select_alone(spj, oracle, field, op, lo, hi):
    import torch
    R, S, _ = spj.generate_host(1 << 17, (1 << 20) + 37, 1.0, seed=5)
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    out = torch.empty_like(dS)
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_select(dS.data_ptr(), S.shape[0], spj.Predicate(field, op, lo, hi), out.data_ptr(),
                                   n.data_ptr(), None))
    torch.cuda.synchronize()
    got = out[:int(n.item())].cpu().numpy().view(np.uint32)
    want = oracle.select(S, field, op, lo, hi)
    assert got.shape == want.shape
    assert np.array_equal(oracle.sort_pairs(got), oracle.sort_pairs(want))


@pytest.mark.parametrize("alg", [0, 1, 2, 3])
def test_join_with_selections(spj, oracle, alg):
    """R keys in a range and S payloads in a range (an S row-id window), for every
    local join, on skewed S (the heavy-key path sees only selected tuples)."""
    R, S, _ = spj.generate_host(1 << 17, 1 << 21, 1.5, seed=6)
    pr = spj.predicate("key", "between", 1000, 90000)
    ps = spj.predicate("payload", "<", 1500000)
    res, logs = run_instance(spj, R, S, join_alg=alg, select_r=pr, select_s=ps, heavy_sample=1 << 14,
                             radix_bits=11 if alg == 0 else 0)
    want = oracle.simple_join(oracle.select(R, 1, 5, 1000, 90000), oracle.select(S, 2, 3, 1500000),
                              keep_unmatched=alg in (2, 3))
    assert same_multiset(oracle, res.pairs(), want)


def test_selections_in_a_batch_and_on_host_slices(spj, oracle):
    import torch
    specs = [(1 << 14, 1 << 16, 0.5), (1 << 16, 1 << 18, 1.2), (3000, 9000, 0.0)]
    data = [spj.generate_host(a, b, z, seed=60 + i) for i, (a, b, z) in enumerate(specs)]
    d = spj.make_design(rank_num=1, select_r=spj.predicate("key", ">=", 100), select_s=spj.predicate("key", "<=",
                                                                                                      40000))
    batch = spj.Batch([a for a, _, _ in specs], [b for _, b, _ in specs], d)
    dR = [torch.from_numpy(R.view(np.int32)).cuda() for R, _, _ in data]
    dS = [torch.from_numpy(S.view(np.int32)).cuda() for _, S, _ in data]
    outs = [torch.empty((batch.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(len(specs))]
    n_out = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    batch.bind([t.data_ptr() for t in dR], [t.data_ptr() for t in dS], [o.data_ptr() for o in outs],
               n_out.data_ptr())
    batch.execute(0)
    torch.cuda.synchronize()
    for j, (R, S, _) in enumerate(data):
        got = outs[j][:int(n_out[j].item())].cpu().numpy().view(np.uint32)
        want = oracle.simple_join(oracle.select(R, 1, 2, 100), oracle.select(S, 1, 1, 40000))
        assert same_multiset(oracle, got, want)
    batch.close()
    # host S of 2^25 tuples: joined in slices that keep R's partitions (selected once)
    R, S, _ = spj.generate_host(1 << 20, 1 << 25, 1.0, seed=66)
    res, _ = run_instance(spj, R, S, select_r=spj.predicate("payload", "between", 5, 700000),
                          select_s=spj.predicate("key", ">", 300))
    want = oracle.simple_join_mt(oracle.select(R, 2, 5, 5, 700000), oracle.select(S, 1, 4, 300))
    assert res.pairs().shape == want.shape
    assert oracle.checksum(res.pairs()) == oracle.checksum(want)


def test_invalid_selection_is_refused(spj):
    with pytest.raises(spj.SpjError, match="selection"):
        spj.Plan(100, 100, spj.make_design(select_r=spj.Predicate(3, 0, 0, 0)))
