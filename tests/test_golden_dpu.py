"""The oracle against golden vectors of the reference's own DPU join kernels
(tests/golden/dpu_kernel_vectors.json, written by make_dpu_vectors.py from
the kernels compiled from the reference tree and run on the host). The inputs
are rebuilt from their parameters (tests/golden/dpu_inputs.py), so these
checks run where the reference tree is absent: every answer the reference's
kernels gave must be the oracle's answer on the same bytes."""
import json
import os
import sys

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import dpu_inputs as di  # noqa: E402

with open(os.path.join(GOLDEN, "dpu_kernel_vectors.json")) as _f:
    V = json.load(_f)


def _ids(cases):
    return [str(c["seed"]) for c in cases]


def test_checksum_is_the_oracles(oracle):
    R, S, _ = oracle.generate(1000, 4000, 1.0, seed=5)
    assert di.checksum(S) == oracle.checksum(S) and di.checksum(R) == oracle.checksum(R)


@pytest.mark.parametrize("c", V["count"], ids=_ids(V["count"]))
def test_count_kernel_vectors(oracle, c):
    T = di.relation(c["seed"], c["n"], (1 << 31) - 1, pad_every=c["pad_every"])
    hist = oracle.partition_count(T, c["P"], c["type"], c["rank_sets"], c["ranks_per_set"])
    assert hist.tolist() == c["hist"]
    assert (np.cumsum(hist) - hist).tolist() == c["start"]


@pytest.mark.parametrize("c", V["chipwise_count"], ids=_ids(V["chipwise_count"]))
def test_chipwise_count_kernel_vectors(oracle, c):
    T = di.relation(c["seed"], c["n"], (1 << 31) - 1, pad_every=c["pad_every"])
    assert oracle.chipwise_partition_count(T, c["ranks"], c["rank_sets"], c["bank_set"]).tolist() == c["hist"]


@pytest.mark.parametrize("c", V["packet"], ids=_ids(V["packet"]))
def test_packet_scatter_vectors(oracle, c):
    T = di.relation(c["seed"], c["n"], (1 << 31) - 1, pad_every=c["pad_every"])
    ranks, G, B = c["ranks"], c["rank_sets"], c["bank_set"]
    if B > 1:
        dest = oracle.chipwise_partition_dest(T, ranks, G, B)
    else:
        dest = oracle.partition_dest(T, 64 * ranks, 0 if G == 1 else 1, G, ranks // G)
    assert di.groups_summary([T[dest == d] for d in range(64 * ranks)]) == c["dest"]


@pytest.mark.parametrize("c", V["align"], ids=_ids(V["align"]))
def test_bank_group_align_vectors(oracle, c):
    T = di.relation(c["seed"], c["n"], (1 << 31) - 1, pad_every=c["pad_every"])
    P = c["ranks_per_set"] * 64 // c["bank_set"]
    dest = oracle.partition_dest(T, P, 0)
    assert di.groups_summary([T[dest == i] for i in range(P)]) == c["groups"]


@pytest.mark.parametrize("c", V["local_partition"], ids=_ids(V["local_partition"]))
def test_local_partition_vectors(oracle, c):
    T = di.relation(c["seed"], c["n"], c["domain"], pad_every=c["pad_every"])
    nz = T[T[:, 0] != 0]
    L = oracle.local_partitions(nz.shape[0])
    assert L == c["L"]
    grouped, off = oracle.local_partition(nz, L)
    assert off.tolist() == c["starts"]
    assert di.groups_summary([grouped[off[p]:off[p + 1]] for p in range(L)]) == c["parts"]


@pytest.mark.parametrize("c", V["join"], ids=_ids(V["join"]))
def test_hash_join_vectors(oracle, c):
    R, S = di.fk_pair(c["seed"], c["n_r"], c["n_s"], c["miss_every"])
    phj = oracle.dpu_phj(R, S)
    assert [int(phj.shape[0]), di.checksum(phj)] == c["phj"] == c["nphj"]
    ref = oracle.simple_join(R, S)
    assert [int(ref.shape[0]), di.checksum(ref)] == c["phj"]


@pytest.mark.parametrize("c", V["nested_loop"], ids=_ids(V["nested_loop"]))
def test_nested_loop_vectors(oracle, c):
    R, S = di.fk_pair(c["seed"], c["n_r"], c["n_s"], c["miss_every"])
    R[:, 1] |= np.uint32(1 << 31)
    rows = oracle.simple_join(R, S, keep_unmatched=True)
    assert [int(rows.shape[0]), di.checksum(rows)] == c["rows"]


@pytest.mark.parametrize("c", V["sort_merge"], ids=_ids(V["sort_merge"]))
def test_sort_merge_vectors(oracle, c):
    elem_range = (c["buckets"] - 1) * c["interval"]
    R, _ = di.fk_pair(c["seed"], elem_range, 1, dense=True)
    pick = (di.stream(c["seed"] + 5, c["n_s"]) % np.uint64(elem_range)).astype(np.int64)
    S = np.stack([R[pick, 0], np.arange(c["n_s"], dtype=np.uint32)], 1).astype(np.uint32)
    # the sort-probe leaves bucket 511 of each full block of 512 and the last bucket unprobed
    B = c["buckets"]
    b = np.minimum(S[:, 0].astype(np.int64) // c["interval"], B - 1)
    loops, rem = divmod(B, 512)
    probed = ((b < loops * 512) & (b % 512 != 511)) | ((b >= loops * 512) & (b - loops * 512 < rem - 1))
    rows = oracle.dpu_smj(R, S[probed])
    assert [int(rows.shape[0]), di.checksum(rows)] == c["rows"]
    assert [int((~probed).sum()), di.checksum(S[~probed])] == c["unprobed"]


@pytest.mark.parametrize("c", V["rank_chain"], ids=_ids(V["rank_chain"]))
def test_rank_chain_vectors(oracle, c):
    R, S = di.fk_pair(c["seed"], c["n_r"], c["n_s"], c["miss_every"])
    sizes_r, sizes_s = oracle.refpipe_dpu_sizes(R, S, ranks=1)
    assert sizes_r.tolist() == c["sizes_r"] and sizes_s.tolist() == c["sizes_s"]
    got = oracle.refpipe_join(R, S, ranks=1)
    assert [int(got.shape[0]), di.checksum(got)] == c["pairs"]
