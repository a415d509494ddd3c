"""GPU tests of the served join stream (spj_server_*): joins submitted together
are batched by the server's worker, and every join's output must equal, as a
pair multiset, the output of the same join run alone through spj_plan_execute,
and carry the generator's exact checksum."""
import threading

import numpy as np
import pytest

from test_gpu_batch import make_batch_inputs as _make_inputs

pytestmark = pytest.mark.gpu


def make_batch_inputs(spj, specs, seed0):
    R, S, exp = _make_inputs(spj, specs, seed0)
    return R, S, [e % (1 << 64) for e in exp]  # the device checksum is read back as a signed int64


MIX = [(1 << 10, 1 << 10, 0.0), (1 << 14, 1 << 16, 1.5), (3000, 24000, 0.5), (1 << 18, 1 << 19, 1.0),
       (1 << 12, 1 << 15, 1.2), (1 << 16, 1 << 16, 0.0), (777, 6216, 0.9), (1 << 17, 1 << 20, 0.3),
       (1 << 11, 1 << 13, 1.5), (1 << 15, 1 << 17, 0.0), (1 << 13, 1 << 13, 0.7), (50000, 400000, 1.4),
       (1 << 10, 1 << 13, 0.0), (1 << 19, 1 << 19, 1.1), (2048, 2048, 1.5), (1 << 16, 1 << 19, 0.2)]


def alone(spj, design, dR, dS, n_r, n_s):
    import torch
    plan = spj.Plan(n_r, n_s, design)
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n.data_ptr(), 0)
    torch.cuda.synchronize()
    plan.close()
    return out[:int(n.item())].cpu().numpy().view(np.uint32)


def serve(spj, server, specs, R, S, threads=1, hold=False):
    """Submits every join (from `threads` client threads), waits for all;
    returns outputs and latencies. With hold, admission is paused until every
    join is queued, so they are batched together."""
    import torch
    outs = [torch.empty((server.output_capacity(n_r, n_s), 2), dtype=torch.int32, device="cuda")
            for n_r, n_s, _ in specs]
    n_out = torch.full((len(specs),), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ids, lat = [None] * len(specs), [None] * len(specs)
    submitted = threading.Barrier(threads + 1)
    if hold:
        server.hold(True)

    def client(k):
        mine = list(range(k, len(specs), threads))
        for j in mine:
            n_r, n_s, _ = specs[j]
            ids[j] = server.submit(R[j].data_ptr(), n_r, S[j].data_ptr(), n_s, outs[j].data_ptr(),
                                   outs[j].shape[0], n_out[j:].data_ptr())
        submitted.wait()
        for j in mine:
            lat[j] = server.wait(ids[j], 60000.0)

    ts = [threading.Thread(target=client, args=(k,)) for k in range(threads)]
    for t in ts:
        t.start()
    submitted.wait()
    if hold:
        server.hold(False)
    for t in ts:
        t.join()
    counts = n_out.cpu().tolist()
    return [outs[j][:counts[j]].cpu().numpy().view(np.uint32) for j in range(len(specs))], lat


@pytest.mark.parametrize("alg", ["phj", "smj", "nl", "nphj"])
@pytest.mark.parametrize("hold", [True, False], ids=["grouped", "streaming"])
def test_served_results_equal_alone_and_in_the_mix(spj, oracle, alg, hold):
    specs = MIX if alg == "phj" else MIX[:8]
    design = spj.make_design(rank_num=1, join_alg=spj.ALG[alg])
    R, S, expect = make_batch_inputs(spj, specs, seed0=300)
    server = spj.Server(hbm_budget_bytes=8 << 30, max_batch=64, streams=4, design=design)
    got, lat = serve(spj, server, specs, R, S, hold=hold)
    st = server.stats()
    server.close()
    for j, (n_r, n_s, _) in enumerate(specs):
        assert got[j].shape == (n_s, 2), (j, got[j].shape)
        assert oracle.checksum(got[j]) == expect[j], j
        want = alone(spj, design, R[j], S[j], n_r, n_s)
        assert np.array_equal(oracle.sort_pairs(got[j]), oracle.sort_pairs(want)), j
    assert st["completed"] == len(specs) and st["failed"] == 0
    if hold:
        assert st["batches"] == 1  # queued while admission was held: one batch of every join
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"] and all(x > 0 for x in lat)


def test_budget_below_one_join_runs_each_alone(spj, oracle):
    specs = MIX[:6]
    design = spj.make_design(rank_num=1)
    R, S, expect = make_batch_inputs(spj, specs, seed0=400)
    server = spj.Server(hbm_budget_bytes=1, max_batch=64, streams=4, design=design)
    got, _ = serve(spj, server, specs, R, S)
    st = server.stats()
    server.close()
    for j in range(len(specs)):
        assert oracle.checksum(got[j]) == expect[j], j
    assert st["batches"] == len(specs) and st["max_inflight_batches"] == 1


def test_budget_bounds_admission(spj, oracle):
    # a budget of about two of the larger joins: batches stay small, results exact
    specs = [(1 << 18, 1 << 19, 1.0)] * 6 + [(1 << 12, 1 << 14, 0.5)] * 6
    design = spj.make_design(rank_num=1)
    R, S, expect = make_batch_inputs(spj, specs, seed0=500)
    probe = spj.Server(1, design=design)
    per_big = 8 * (3 << 18) + 8 * probe.output_capacity(1 << 18, 1 << 19) + 16 * (3 << 18)
    probe.close()
    budget = 2 * per_big + (8 << 20)
    server = spj.Server(hbm_budget_bytes=budget, max_batch=64, streams=4, design=design)
    got, _ = serve(spj, server, specs, R, S, hold=True)
    st = server.stats()
    server.close()
    for j in range(len(specs)):
        assert oracle.checksum(got[j]) == expect[j], j
    assert st["hbm_peak_bytes"] <= budget + (64 << 20)
    assert st["batches"] >= 3


def test_concurrent_clients(spj, oracle):
    specs = MIX
    design = spj.make_design(rank_num=1)
    R, S, expect = make_batch_inputs(spj, specs, seed0=600)
    server = spj.Server(hbm_budget_bytes=8 << 30, max_batch=8, streams=3, design=design)
    got, _ = serve(spj, server, specs, R, S, threads=4)
    st = server.stats()
    server.reset_stats()
    assert server.stats()["completed"] == 0
    server.close()
    for j in range(len(specs)):
        assert oracle.checksum(got[j]) == expect[j], j
    assert st["completed"] == len(specs) and st["mean_batch"] <= 8


def test_server_argument_errors(spj):
    import torch
    server = spj.Server(1 << 30, design=spj.make_design(rank_num=1))
    d = torch.zeros((64, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(spj.SpjError, match="capacity"):
        server.submit(d.data_ptr(), 16, d.data_ptr(), 16, d.data_ptr(), 16, n.data_ptr())
    with pytest.raises(spj.SpjError, match="aligned"):
        server.submit(d.data_ptr() + 8, 16, d.data_ptr(), 16, d.data_ptr(), 1 << 30, n.data_ptr())
    with pytest.raises(spj.SpjError, match="unknown"):
        server.wait(12345, 10.0)
    server.close()
