"""The multi-GPU join's exchange protocol on CPU: two and three gloo ranks run
spidjoin.DistributedJoin with host stand-ins for the device split and the local
join (the oracle's hash and join -- test scaffolding only), and the union of the
ranks' outputs must equal the join of the union of the shards. Every rank must
receive exactly the keys whose destination it is."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dest(keys, world):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    h = oracle.glb_partition_hash_np(keys).astype(np.uint64)
    return ((h * np.uint64(world)) >> np.uint64(32)).astype(np.int64)


def _dataset(seed, n_r, n_s, hot=0.0):
    rng = np.random.default_rng(seed)
    keys = rng.permutation(n_r).astype(np.uint32) + 1
    keys[:3] = [0x80000001, 0xFFFFFF00, 0x7FFFFFFF]  # keys above 2^31 too
    R = np.stack([keys, np.arange(n_r, dtype=np.uint32)], axis=1)
    sk = keys[rng.integers(0, n_r, n_s)]
    if hot:  # two hot keys carry a share `hot` of S each
        sk[rng.random(n_s) < hot] = keys[1]
        sk[rng.random(n_s) < hot] = keys[7]
    sk[rng.random(n_s) < 0.05] = 0                       # padding
    miss = rng.random(n_s) < 0.05
    sk[miss] = (n_r + 1 + rng.integers(0, 1000, int(miss.sum()))).astype(np.uint32)  # no partner
    S = np.stack([sk, np.arange(n_s, dtype=np.uint32)], axis=1)
    return R, S


def _rank_main(rank, world, port, seed, out_q, hot=0.0):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "spid-join_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import spidjoin
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        R, S = _dataset(seed, 5000, 20000, hot)
        # uneven shards: rank i holds a contiguous slice of each relation
        rb = np.linspace(0, R.shape[0], world + 1).astype(int)
        sb = (np.linspace(0, 1, world + 1) ** 1.5 * S.shape[0]).astype(int)
        myR, myS = R[rb[rank]:rb[rank + 1]], S[sb[rank]:sb[rank + 1]]

        def split(T, heavy, mode):
            a = T.numpy().view(np.uint32).reshape(-1, 2)
            a = a[a[:, 0] != 0]
            d = _dest(a[:, 0], world)
            hv = np.isin(a[:, 0], np.array(heavy, dtype=np.uint32))
            if mode == 1:
                d[hv] = rank
            elif mode == 2:
                a, d = a[~hv], d[~hv]
            order = np.argsort(d, kind="stable")
            counts = np.bincount(d, minlength=world).astype(np.int64)
            return torch.from_numpy(a[order].view(np.int32).copy()), torch.from_numpy(counts)

        received = {}

        def join(Rr, Sr):
            received["R"], received["S"] = Rr.numpy().view(np.uint32), Sr.numpy().view(np.uint32)
            out = oracle.simple_join(received["R"], received["S"])
            return torch.from_numpy(out.view(np.int32).copy()), torch.tensor([out.shape[0]])

        dj = spidjoin.DistributedJoin(split=split, join=join)
        pairs, n = dj.run(torch.from_numpy(myR.view(np.int32).copy()), torch.from_numpy(myS.view(np.int32).copy()))
        heavy = np.array(dj.last_heavy, dtype=np.uint32)
        hr = np.isin(received["R"][:, 0], heavy)
        hs = np.isin(received["S"][:, 0], heavy)
        ok_dest = (bool(np.all(_dest(received["R"][~hr, 0], world) == rank)) and
                   bool(np.all(_dest(received["S"][~hs, 0], world) == rank)) and
                   int(hr.sum()) == len(heavy) and  # every rank holds every heavy key's R tuple
                   np.array_equal(np.sort(received["S"][hs, 1]), np.sort(myS[np.isin(myS[:, 0], heavy), 1])))
        out_q.put((rank, pairs[:int(n[0])].numpy().view(np.uint32).copy(), ok_dest,
                   received["R"].shape[0] - int(hr.sum()), received["S"].shape[0], dj.last_heavy))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,hot", [(2, 0.0), (3, 0.0), (3, 0.2), (2, 0.3)])
def test_exchange_then_local_joins_equal_global_join(oracle, world, hot):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, 7, q, hot)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    R, S = _dataset(7, 5000, 20000, hot)
    want = oracle.sort_pairs(oracle.simple_join(R, S))
    got = oracle.sort_pairs(np.concatenate([r[1] for r in res]))
    assert np.array_equal(got, want)
    assert all(r[2] for r in res), "a rank received keys of another destination"
    heavy = res[0][5]
    assert all(r[5] == heavy for r in res)  # every rank computed the same heavy list
    assert (len(heavy) >= 2) == (hot > 0)
    assert sum(r[3] for r in res) == int((R[:, 0] != 0).sum()) - len(heavy)
    assert sum(r[4] for r in res) == int((S[:, 0] != 0).sum())


def test_exchange_layout_tiles_every_receive_buffer():
    sys.path.insert(0, os.path.join(ROOT, "spid-join_b200"))
    import spidjoin
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        C = rng.integers(0, 1000, (world, world)).tolist()
        C[0][world - 1] = 0
        layouts = [spidjoin.exchange_layout(C, r) for r in range(world)]
        need = max(sum(C[s][d] for s in range(world)) for d in range(world))
        for d in range(world):
            segs = sorted((layouts[s][1][d], layouts[s][1][d] + C[s][d]) for s in range(world))
            pos = 0
            for a, b in segs:  # senders' segments follow each other without gaps or overlap
                assert a == pos
                pos = b
            assert pos == layouts[d][0] <= need == layouts[0][2]


def _rank_fail_main(rank, world, port, out_q, failure="raise"):
    """Rank 1 fails on the host before its first exchange: its split raises and
    it leaves (failure "raise"), or it stalls there without leaving (failure
    "stall"). Rank 0 runs normally and must end with an error, not wait for
    good: at once when its peer's connection drops, at the process group's 3 s
    timeout when the peer stalls."""
    import datetime
    import time

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "spid-join_b200"))
    import spidjoin
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    R, S = _dataset(11, 2000, 8000)

    def split(T, heavy, mode):
        if rank == 1:
            if failure == "stall":
                time.sleep(7)  # does not reach the exchange before rank 0's timeout
            raise RuntimeError("injected failure on rank 1")
        a = T.numpy().view(np.uint32).reshape(-1, 2)
        a = a[a[:, 0] != 0]
        d = _dest(a[:, 0], world)
        order = np.argsort(d, kind="stable")
        return torch.from_numpy(a[order].view(np.int32).copy()), torch.from_numpy(np.bincount(d, minlength=world))

    dj = spidjoin.DistributedJoin(split=split, join=lambda r, s: (r, torch.tensor([0])), heavy=False)
    t0 = time.monotonic()
    try:
        dj.run(torch.from_numpy(R.view(np.int32).copy()), torch.from_numpy(S.view(np.int32).copy()))
        out_q.put((rank, "finished", "", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001 -- the outcome is what the test checks
        out_q.put((rank, type(e).__name__, str(e)[:200], time.monotonic() - t0))
    # the group is broken: leave without another collective, once the result is sent
    out_q.close()
    out_q.join_thread()
    os._exit(0)


@pytest.mark.parametrize("failure", ["raise", "stall"])
def test_a_failing_rank_ends_its_peers_with_an_error(failure):
    """Failure detection on the host: when one rank raises before its exchange
    and leaves, or stalls there, the other rank's pending collective ends with
    an error (within the process group's timeout) instead of waiting for
    good."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_fail_main, args=(r, 2, port, q, failure)) for r in range(2)]
    for p in procs:
        p.start()
    res = {r: (kind, msg, secs) for r, kind, msg, secs in (q.get(timeout=120) for _ in range(2))}
    for p in procs:
        p.join(60)
        assert p.exitcode == 0, "a rank did not exit"
    assert res[1][0] == "RuntimeError" and "injected failure" in res[1][1]
    assert res[0][0] != "finished", "rank 0 finished a join its peer never joined"
    assert res[0][2] < (2 if failure == "raise" else 6.5)
    if failure == "stall":
        assert res[0][2] >= 2.5, "rank 0 ended before its process group's timeout"
