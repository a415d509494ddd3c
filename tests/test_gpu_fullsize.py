"""GPU parity at the benchmark's full sizes, where the oracle would take too long:
size-independent properties through the C ABI. The seeded generator knows every S
tuple's R row when it makes it, so it returns the exact answer's pair count (|S|:
every S key is in R) and order-independent checksum; each join must reproduce both,
twice in a row on the same plan (idempotence).

* config 2: |R| = 2^27, |S| = 2^29, Zipf 1.0, replication groups of 4 (-r 4 -R 4 -B 1);
* config 3: |R| = 2^26, |S| = 2^29, Zipf 1.5, with the hash, non-partitioned hash,
  sort-merge and nested-loop local joins, and fixed replication groups of 1, 4 and 16;
* config 4: the 256-join mix (|R| log-uniform in [2^12, 2^24], R:S in {1, 2, 4, 8},
  Zipf in [0, 1.5]) as one batch, every join checked.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x5EED5EED


def _device_inputs(spj, n_r, n_s, zipf, seed):
    import torch
    dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
    dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
    expect = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_generate_device(seed, n_r, n_s, zipf, dR.data_ptr(), dS.data_ptr(), expect.data_ptr(),
                                            None))
    torch.cuda.synchronize()
    return dR, dS, int(expect.item())


def _join_twice(spj, dR, dS, design):
    """Runs the plain join twice on one plan; returns [(pairs, checksum)] per run."""
    import torch
    n_r, n_s = dR.shape[0], dS.shape[0]
    plan = spj.Plan(n_r, n_s, design)
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    csum = torch.zeros(1, dtype=torch.int64, device="cuda")
    got = []
    for _ in range(2):
        plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n_out.data_ptr(), None)
        spj.check(spj.lib().spj_checksum_device(out.data_ptr(), n_out.data_ptr(), csum.data_ptr(), None))
        torch.cuda.synchronize()
        got.append((int(n_out.item()), int(csum.item())))
    plan.stats()  # raises if a device-side capacity check fired
    plan.close()
    del out
    return got


@pytest.fixture
def free_cache():
    yield
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def test_config2_full_size(spj, free_cache):
    n_r, n_s = 1 << 27, 1 << 29
    dR, dS, expect = _device_inputs(spj, n_r, n_s, 1.0, SEED)
    d = spj.make_design(rank_num=4, rank_set=4, bank_set=1)
    assert _join_twice(spj, dR, dS, d) == [(n_s, expect)] * 2


@pytest.fixture(scope="module")
def config3(spj):
    yield _device_inputs(spj, 1 << 26, 1 << 29, 1.5, SEED + 3)
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("alg", ["phj", "nphj", "smj", "nl"])
def test_config3_full_size_each_local_join(spj, config3, alg, free_cache):
    dR, dS, expect = config3
    d = spj.make_design(rank_num=4, rank_set=4, bank_set=1, join_alg=alg)
    assert _join_twice(spj, dR, dS, d) == [(dS.shape[0], expect)] * 2


@pytest.mark.parametrize("groups", [1, 4, 16])
def test_config3_full_size_fixed_replication_groups(spj, config3, groups, free_cache):
    # every partition built by `groups` units, its S split among them (-R groups)
    dR, dS, expect = config3
    d = spj.make_design(rank_num=groups, rank_set=groups, bank_set=1, skew_mode=1)
    assert _join_twice(spj, dR, dS, d) == [(dS.shape[0], expect)] * 2


def test_config4_full_scale_batch(spj, free_cache):
    import torch
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import c4_specs
    specs = c4_specs()
    assert len(specs) == 256
    R, S, exp = [], [], []
    for i, (n_r, n_s, z) in enumerate(specs):
        dR, dS, e = _device_inputs(spj, n_r, n_s, z, SEED + 1000 + i)
        R.append(dR)
        S.append(dS)
        exp.append(e)
    b = spj.Batch([x[0] for x in specs], [x[1] for x in specs], spj.make_design(rank_num=1))
    outs = [torch.empty((b.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(len(specs))]
    n_out = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    b.bind([t.data_ptr() for t in R], [t.data_ptr() for t in S], [o.data_ptr() for o in outs], n_out.data_ptr())
    cs = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    for _ in range(2):
        b.execute(None)
        for j, o in enumerate(outs):
            spj.check(spj.lib().spj_checksum_device(o.data_ptr(), n_out[j:].data_ptr(), cs[j:].data_ptr(), None))
        torch.cuda.synchronize()
        assert n_out.cpu().numpy().tolist() == [x[1] for x in specs]
        got = cs.cpu().numpy().astype(np.uint64).tolist()
        assert got == [e % (1 << 64) for e in exp]
    b.close()


def test_c2_pairs_equal_oracle_byte_for_byte(spj, oracle, free_cache):
    """Config 2 in full (2^27 R x 2^29 S, Zipf 1.0, -r 4 -R 4 -B 1) through the C
    ABI: the pairs, copied to the host, equal the oracle's independent join byte
    for byte after the canonical sort (ascending (R payload, S payload)); count
    and checksum are checked beside it. The oracle's threaded join and sort give
    the same bytes as its single-threaded ones (a CPU test pins that)."""
    import time
    import torch
    n_r, n_s = 1 << 27, 1 << 29
    t0 = time.time()
    dR, dS, expect = _device_inputs(spj, n_r, n_s, 1.0, SEED)
    plan = spj.Plan(n_r, n_s, spj.make_design(rank_num=4, rank_set=4, bank_set=1))
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n_out.data_ptr(), None)
    torch.cuda.synchronize()
    plan.stats()
    plan.close()
    k = int(n_out.item())
    got = out[:k].cpu().numpy().view(np.uint32)
    R = dR.cpu().numpy().view(np.uint32)
    S = dS.cpu().numpy().view(np.uint32)
    del out, dR, dS
    torch.cuda.empty_cache()
    t_gpu = time.time() - t0
    want = oracle.simple_join_mt(R, S)
    del R, S
    assert k == want.shape[0] == n_s
    assert oracle.checksum(got) == oracle.checksum(want) == expect & (2**64 - 1)
    oracle.sort_pairs_mt(got, inplace=True)
    oracle.sort_pairs_mt(want, inplace=True)
    assert np.array_equal(got, want)
    print(f"c2 byte-for-byte: {k} pairs; device part {t_gpu:.1f} s, oracle and sorts {time.time() - t0 - t_gpu:.1f} s")
