"""Writes dpu_kernel_vectors.json: answers of the reference's own DPU join
kernels (src/dpu/src/join/ of yonsei-hpcp/spid-join, compiled from the
reference tree by `make -C oracle ref` and run on the host through
oracle/dpu_ref.py) on the deterministic inputs of dpu_inputs.py. With them the
oracle's agreement with the reference's kernels is checked where the
reference tree is absent (tests/test_golden_dpu.py). Needs the built runners;
the inputs are stored as their parameters, the answers as counts and
order-independent checksums (full histograms for the counts)."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import dpu_inputs as di  # noqa: E402
import dpu_ref  # noqa: E402


def _split_blocks(T, D):
    per = (T.shape[0] * 8 + (D * 8 - T.shape[0] * 8 % (D * 8))) // 8 // D
    padded = np.zeros((per * D, 2), dtype=np.uint32)
    padded[:T.shape[0]] = T
    return [padded[b * per:(b + 1) * per] for b in range(D)]


def count_cases():
    out = []
    for seed, n, P, type_, G, rps in [(11, 50001, 64, 0, 1, 1), (12, 40000, 256, 1, 4, 1), (13, 30000, 1024, 0, 1, 1),
                                      (14, 20001, 2048, 1, 2, 16)]:
        T = di.relation(seed, n, (1 << 31) - 1, pad_every=37)
        hist, start = dpu_ref.partition_count(T, P, type_, G, rps)
        out.append(dict(seed=seed, n=n, P=P, type=type_, rank_sets=G, ranks_per_set=rps, pad_every=37,
                        hist=hist.tolist(), start=start.tolist()))
    return out


def chipwise_count_cases():
    out = []
    for seed, n, ranks, G, B in [(21, 30001, 1, 1, 8), (22, 25000, 8, 2, 32)]:
        T = di.relation(seed, n, (1 << 31) - 1, pad_every=41)
        hist, _ = dpu_ref.chipwise_partition_count(T, ranks, G, B)
        out.append(dict(seed=seed, n=n, ranks=ranks, rank_sets=G, bank_set=B, pad_every=41, hist=hist.tolist()))
    return out


def packet_cases():
    out = []
    for seed, n, ranks, G, dpu, ps, B in [(31, 20001, 1, 1, 0, 8, 1), (32, 15000, 4, 2, 19, 16, 1),
                                          (33, 18000, 4, 1, 42, 32, 16)]:
        T = di.relation(seed, n, (1 << 31) - 1, pad_every=53)
        groups = dpu_ref.packet_scatter(T, ranks, G, dpu, ps, bank_set=B)
        out.append(dict(seed=seed, n=n, ranks=ranks, rank_sets=G, dpu_id=dpu, packet_size=ps, bank_set=B,
                        pad_every=53, dest=di.groups_summary(groups)))
    return out


def align_cases():
    out = []
    for seed, n, rps, B in [(41, 30001, 4, 16), (42, 12000, 1, 8)]:
        T = di.relation(seed, n, (1 << 31) - 1, pad_every=29)
        groups = dpu_ref.bg_broadcast_align(T, rps, B)
        out.append(dict(seed=seed, n=n, ranks_per_set=rps, bank_set=B, pad_every=29, groups=di.groups_summary(groups)))
    return out


def local_partition_cases():
    out = []
    for seed, n in [(51, 30000), (52, 1936)]:
        T = di.relation(seed, n, 4 * n, pad_every=41)
        grouped, starts, L = dpu_ref.local_partition(T)
        parts = [grouped[starts[p]:starts[p + 1]] for p in range(L)]
        out.append(dict(seed=seed, n=n, domain=4 * n, pad_every=41, L=int(L), starts=starts.tolist(),
                        parts=di.groups_summary(parts)))
    return out


def join_cases():
    out = []
    for seed, n_r, n_s, miss in [(61, 20000, 70000, 9), (62, 1 << 15, 1 << 17, 0)]:
        R, S = di.fk_pair(seed, n_r, n_s, miss)
        rg, ro, L = dpu_ref.local_partition(R)
        sg, so, _ = dpu_ref.local_partition(S, partitions=L)
        phj = dpu_ref.hash_join(rg, ro, sg, so)
        nphj, _ = dpu_ref.nphj(R, S)
        out.append(dict(seed=seed, n_r=n_r, n_s=n_s, miss_every=miss,
                        phj=[int(phj.shape[0]), di.checksum(phj)], nphj=[int(nphj.shape[0]), di.checksum(nphj)]))
    return out


def nested_loop_cases():
    out = []
    for seed, n_r, n_s, miss in [(71, 2000, 2500, 5), (72, 700, 3000, 0)]:
        R, S = di.fk_pair(seed, n_r, n_s, miss)
        R[:, 1] |= np.uint32(1 << 31)  # payloads above every key: the kernel's second rewrite cannot occur
        rows = dpu_ref.nested_loop(R, S)
        out.append(dict(seed=seed, n_r=n_r, n_s=n_s, miss_every=miss, rows=[int(rows.shape[0]), di.checksum(rows)]))
    return out


def sort_merge_cases():
    out = []
    for seed, B, interval, n_s in [(81, 513, 64, 20000), (82, 1024, 64, 40000)]:
        elem_range = (B - 1) * interval
        R, _ = di.fk_pair(seed, elem_range, 1, dense=True)
        pick = (di.stream(seed + 5, n_s) % np.uint64(elem_range)).astype(np.int64)
        S = np.stack([R[pick, 0], np.arange(n_s, dtype=np.uint32)], 1).astype(np.uint32)
        rows, unprobed = dpu_ref.sort_merge(R, S, elem_range, interval)
        out.append(dict(seed=seed, buckets=B, interval=interval, n_s=n_s, rows=[int(rows.shape[0]), di.checksum(rows)],
                        unprobed=[int(unprobed.shape[0]), di.checksum(unprobed)]))
    return out


def rank_chain_cases():
    """The hash join over one rank of 64 DPUs by the reference's kernels
    alone (count, packet scatter, exchange, local partitioning, build, probe)."""
    out = []
    for seed, n_r, n_s in [(91, 1 << 15, 1 << 17)]:
        R, S = di.fk_pair(seed, n_r, n_s, 13)
        D = 64
        to_r = [dpu_ref.packet_scatter(b, 1, 1, i) for i, b in enumerate(_split_blocks(R, D))]
        to_s = [dpu_ref.packet_scatter(b, 1, 1, i) for i, b in enumerate(_split_blocks(S, D))]
        sizes_r, sizes_s, pairs = [], [], []
        for d in range(D):
            r_d = np.concatenate([to_r[b][d] for b in range(D)])
            s_d = np.concatenate([to_s[b][d] for b in range(D)])
            sizes_r.append(int(r_d.shape[0]))
            sizes_s.append(int(s_d.shape[0]))
            rg, ro, L = dpu_ref.local_partition(r_d)
            sg, so, _ = dpu_ref.local_partition(s_d, partitions=L)
            pairs.append(dpu_ref.hash_join(rg, ro, sg, so))
        got = np.concatenate(pairs)
        out.append(dict(seed=seed, n_r=n_r, n_s=n_s, miss_every=13, sizes_r=sizes_r, sizes_s=sizes_s,
                        pairs=[int(got.shape[0]), di.checksum(got)]))
    return out


def main():
    if not dpu_ref.available():
        sys.exit("the reference's DPU kernels are not built: make -C oracle ref")
    doc = {
        "source": "yonsei-hpcp/spid-join src/dpu/src/join/*.c run on the host by oracle/dpu_ref.py",
        "count": count_cases(), "chipwise_count": chipwise_count_cases(), "packet": packet_cases(),
        "align": align_cases(), "local_partition": local_partition_cases(), "join": join_cases(),
        "nested_loop": nested_loop_cases(), "sort_merge": sort_merge_cases(), "rank_chain": rank_chain_cases(),
    }
    with open(os.path.join(HERE, "dpu_kernel_vectors.json"), "w") as f:
        json.dump(doc, f, separators=(",", ":"))
        f.write("\n")


if __name__ == "__main__":
    main()
