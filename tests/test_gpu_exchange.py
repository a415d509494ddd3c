"""GPU tests of the multi-GPU join's pieces that one GPU can run: the device
split by destination rank (spj_exchange_split) against the oracle's hash, and
DistributedJoin end to end on a one-rank NCCL group."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dest(oracle, keys, world):
    h = oracle.glb_partition_hash_np(keys).astype(np.uint64)
    return ((h * np.uint64(world)) >> np.uint64(32)).astype(np.int64)


@pytest.mark.parametrize("world", [1, 2, 5, 8, 1024])
def test_exchange_split_groups_by_destination(spj, oracle, world):
    import torch
    n_r, n_s = 1 << 16, (1 << 20) + 3
    R, S, _ = spj.generate_host(n_r, n_s, 1.2, seed=5)
    S = S.copy()
    S[::97, 0] = 0  # padding is dropped
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    out = torch.empty_like(dS)
    cnt = torch.empty(2 * world, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_exchange_split(dS.data_ptr(), n_s, world, 0, None, 0, 0, out.data_ptr(), cnt.data_ptr(),
                                           None))
    torch.cuda.synchronize()
    counts = cnt[:world].cpu().numpy()
    keep = S[S[:, 0] != 0]
    d = _dest(oracle, keep[:, 0], world)
    assert np.array_equal(counts, np.bincount(d, minlength=world))
    got = out.cpu().numpy().view(np.uint32)[:keep.shape[0]]
    off = np.concatenate([[0], np.cumsum(counts)])
    for r in range(world):
        seg = got[off[r]:off[r + 1]]
        assert np.all(_dest(oracle, seg[:, 0], world) == r)
        assert np.array_equal(oracle.sort_pairs(seg), oracle.sort_pairs(keep[d == r]))


@pytest.mark.parametrize("fused", [False, True])
def test_distributed_join_heavy_keys_one_rank(spj, oracle, fused):
    # Zipf 1.5: the top key is ~38% of S, so the heavy-key path (S kept, R
    # replicated through the all-gather) runs even with one rank
    import torch
    import torch.distributed as dist
    # one rank: an in-process store, no TCP rendezvous (a freed port can be taken again)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        n_r, n_s = 1 << 17, 1 << 20
        R, S, expect = spj.generate_host(n_r, n_s, 1.5, seed=23)
        dj = spj.DistributedJoin(design=spj.make_design(rank_num=1), fused=fused, heavy="always")
        pairs, n = dj.run(torch.from_numpy(R.view(np.int32)).cuda(), torch.from_numpy(S.view(np.int32)).cuda())
        torch.cuda.synchronize()
        got = pairs[:int(n.item())].cpu().numpy().view(np.uint32)
        assert len(dj.last_heavy) >= 1
        assert got.shape == (n_s, 2) and oracle.checksum(got) == expect
        dj.close()
    finally:
        dist.destroy_process_group()


def test_distributed_join_one_rank(spj, oracle):
    import torch
    import torch.distributed as dist
    # one rank: an in-process store, no TCP rendezvous (a freed port can be taken again)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1)
    try:
        n_r, n_s = 1 << 18, 1 << 20
        R, S, expect = spj.generate_host(n_r, n_s, 1.0, seed=9)
        dj = spj.DistributedJoin(design=spj.make_design(rank_num=1))
        dR = torch.from_numpy(R.view(np.int32)).cuda()
        dS = torch.from_numpy(S.view(np.int32)).cuda()
        for _ in range(2):
            pairs, n = dj.run(dR, dS)
            torch.cuda.synchronize()
            got = pairs[:int(n.item())].cpu().numpy().view(np.uint32)
            assert got.shape == (n_s, 2)
            assert oracle.checksum(got) == expect
        dj.close()
    finally:
        dist.destroy_process_group()


def test_fused_scatter_into_several_receive_buffers(spj, oracle):
    # four ranks emulated on one GPU: each shard is scattered straight into the
    # four receive buffers at the offsets of the size matrix, then every
    # "rank" joins what it received; the union is the global join
    import torch
    world = 4
    n_r, n_s = 1 << 16, 1 << 18
    R, S, expect = spj.generate_host(n_r, n_s, 1.1, seed=21)
    shards = {"R": np.array_split(R, world), "S": np.array_split(S, world)}
    recv = {}
    for rel in ("R", "S"):
        dev = [torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda() for x in shards[rel]]
        C = []
        for t in dev:
            c = torch.empty(world, dtype=torch.int64, device="cuda")
            spj.check(spj.lib().spj_exchange_count(t.data_ptr(), t.shape[0], world, 0, None, 0, 0, c.data_ptr(), None))
            C.append(c.tolist())
        bufs = [torch.empty((spj.exchange_layout(C, d)[2] + 8, 2), dtype=torch.int32, device="cuda")
                for d in range(world)]
        ptrs = torch.tensor([b.data_ptr() for b in bufs], dtype=torch.int64, device="cuda")
        for src, t in enumerate(dev):
            offs = torch.tensor(spj.exchange_layout(C, src)[1], dtype=torch.int64, device="cuda")
            cur = torch.empty(world, dtype=torch.int64, device="cuda")
            spj.check(spj.lib().spj_exchange_scatter(t.data_ptr(), t.shape[0], world, src, None, 0, 0, ptrs.data_ptr(),
                                                     offs.data_ptr(), cur.data_ptr(), None))
        torch.cuda.synchronize()
        recv[rel] = [bufs[d][:spj.exchange_layout(C, d)[0]].cpu().numpy().view(np.uint32) for d in range(world)]
        whole = np.concatenate(shards[rel])
        dest = _dest(oracle, whole[:, 0], world)
        for d in range(world):
            assert np.all(_dest(oracle, recv[rel][d][:, 0], world) == d)
            assert np.array_equal(oracle.sort_pairs(recv[rel][d]), oracle.sort_pairs(whole[dest == d]))
    out = np.concatenate([oracle.simple_join(recv["R"][d], recv["S"][d]) for d in range(world)])
    assert out.shape == (n_s, 2) and oracle.checksum(out) == expect


def test_distributed_join_fused_one_rank(spj, oracle):
    import torch
    import torch.distributed as dist
    # one rank: an in-process store, no TCP rendezvous (a freed port can be taken again)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        n_r, n_s = 1 << 18, 1 << 20
        R, S, expect = spj.generate_host(n_r, n_s, 1.0, seed=19)
        dj = spj.DistributedJoin(design=spj.make_design(rank_num=1), fused=True)
        dR = torch.from_numpy(R.view(np.int32)).cuda()
        dS = torch.from_numpy(S.view(np.int32)).cuda()
        for _ in range(2):
            pairs, n = dj.run(dR, dS)
            torch.cuda.synchronize()
            got = pairs[:int(n.item())].cpu().numpy().view(np.uint32)
            assert got.shape == (n_s, 2) and oracle.checksum(got) == expect
        dj.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", [1, 2])
def test_exchange_split_routes_heavy_keys(spj, oracle, mode):
    # heavy keys (sorted, unsigned): with mode 1 their tuples stay on rank `me`,
    # with mode 2 they leave the exchange; every other tuple goes by the hash
    import torch
    world, me, n = 6, 4, 1 << 18
    rng = np.random.default_rng(31)
    keys = rng.integers(1, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    heavy = np.array(sorted({int(keys[5]), int(keys[77]), 0xFFFFFFF0, int(keys[1000])}), dtype=np.uint32)
    keys[rng.random(n) < 0.3] = keys[5]
    keys[::50] = 0xFFFFFFF0
    T = np.stack([keys, np.arange(n, dtype=np.uint32)], axis=1)
    dT = torch.from_numpy(T.view(np.int32)).cuda()
    dH = torch.from_numpy(heavy.view(np.int32)).cuda()
    out = torch.empty_like(dT)
    cnt = torch.empty(2 * world, dtype=torch.int64, device="cuda")
    spj.check(spj.lib().spj_exchange_split(dT.data_ptr(), n, world, me, dH.data_ptr(), len(heavy), mode,
                                           out.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    d = _dest(oracle, T[:, 0], world)
    hv = np.isin(T[:, 0], heavy)
    keep = np.ones(n, dtype=bool)
    if mode == 1:
        d[hv] = me
    else:
        keep = ~hv
    counts = cnt[:world].cpu().numpy()
    assert np.array_equal(counts, np.bincount(d[keep], minlength=world))
    got = out.cpu().numpy().view(np.uint32)[:int(counts.sum())]
    off = np.concatenate([[0], np.cumsum(counts)])
    for r in range(world):
        want = T[keep & (d == r)]
        assert np.array_equal(oracle.sort_pairs(got[off[r]:off[r + 1]]), oracle.sort_pairs(want))


@pytest.mark.parametrize("heavy", [0, 2])
def test_sharded_join_native_one_rank(spj, oracle, heavy):
    # the library's own NCCL driver (spj_dist_*) on a one-rank communicator:
    # heavy=2 runs the heavy-key sample, the replicated R rows and both
    # exchange modes even with one rank; the pairs equal the oracle's join
    import torch
    n_r, n_s = 1 << 17, 1 << 20
    R, S, expect = spj.generate_host(n_r, n_s, 1.5, seed=29)
    sj = spj.ShardedJoin(world=1, rank=0, design=spj.make_design(rank_num=1), heavy=heavy)
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    want = oracle.sort_pairs(oracle.simple_join(R, S))
    for _ in range(2):  # the second call reuses the handle's plan and buffers
        pairs, n = sj.run(dR, dS)
        got = pairs.cpu().numpy().view(np.uint32)
        assert n == n_s and oracle.checksum(got) == expect
        assert np.array_equal(oracle.sort_pairs(got), want)
    assert (len(sj.last_heavy) >= 1) == (heavy == 2)
    assert sj.last_heavy == sorted(sj.last_heavy)
    sj.close()


def test_sharded_join_native_ragged_and_empty(spj, oracle):
    import torch
    sj = spj.ShardedJoin(world=1, rank=0, heavy=2)
    R, S, _ = spj.generate_host(1000, 7777, 1.2, seed=31)
    S = S.copy()
    S[::5, 0] = 0  # padding never joins
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    for r, s, hr, hs in ((dR, dS, R, S), (dR[:0], dS, R[:0], S), (dR, dS[:0], R, S[:0]), (dR[:0], dS[:0], R[:0], S[:0])):
        pairs, n = sj.run(r, s)
        want = oracle.sort_pairs(oracle.simple_join(hr, hs))
        assert n == want.shape[0]
        assert np.array_equal(oracle.sort_pairs(pairs.cpu().numpy().view(np.uint32)), want)
    sj.close()


def test_sharded_join_native_abort(spj):
    """After spj_dist_abort the handle refuses joins (SPJ_E_STATE) and can still
    be destroyed; a world of one has no peer to wait for."""
    import torch
    sj = spj.ShardedJoin(world=1, rank=0)
    R, S, _ = spj.generate_host(4096, 8192, 0.0, seed=3)
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    _, n = sj.run(dR, dS)
    assert n == 8192
    sj.abort()
    sj.abort()  # a second abort is a no-op
    with pytest.raises(spj.SpjError, match="STATE"):
        sj.run(dR, dS)
    sj.close()
