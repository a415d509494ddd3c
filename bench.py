#!/usr/bin/env python
"""Benchmark of the B200 SPID-Join equi-join: join tuples/s (|R|+|S|) and the
fraction of the HBM roofline, on the seeded synthetic relations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl ours|reference]

One step = one plain join (partition, build, probe, compaction) of the workload
with R and S resident in HBM. Rank 0 prints one JSON line. Under torchrun with
N > 1 the step is one join sharded over the N GPUs (each rank holds the
workload's |R| and |S|: weak scaling): split by destination rank, exchange of R
and S (`--exchange fused`, the default: a scatter straight into the peers'
receive buffers; `nccl`: NCCL all-to-all), local join; the time is the max over
ranks (`--replicas`: N independent joins instead).
Workloads: c1, c2 (default), c3, their uniform/skewed twins, c4 (batched), c5
(served stream); `--alg` picks the local join (0 hash, 1 non-partitioned hash,
2 sort-merge, 3 nested loop), `--groups G` the replication groups (-r G -R G
-B 1), `--skew 1` fixed instead of adaptive replication.
The default c2 line also carries, measured on the same GPU with every leg
checked (`--no-extra` skips them): `skew` (the c2 shape uniform against Zipf
1.5), `batched` (config 4 as one batch against one plan per join), `c1` (the
reference driver's own config 1) and `sort_merge` (config 3 with the sort-merge
against the hash local join).
`--impl reference` times the reference's algorithm restated on the host cores
(the oracle's pipeline restatement; the UPMEM original cannot run here).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "spid-join_b200"))

WORKLOADS = {
    # name: |R|, |S|, zipf, (ranks, rank sets, bank set), description
    "c1": (1 << 20, 1 << 21, 0.0, (1, 1, 1), "plain equi-join |R|=2^20 |S|=2^21 uniform (-s 1048576 -t 2 -z 0 -r 1)"),
    "c2": (1 << 27, 1 << 29, 1.0, (4, 4, 1),
           "plain equi-join |R|=2^27 |S|=2^29 Zipf 1.0, replication groups of 4 (-r 4 -R 4 -B 1)"),
    "c3": (1 << 26, 1 << 29, 1.5, (4, 4, 1), "plain equi-join |R|=2^26 |S|=2^29 Zipf 1.5, groups of 4"),
    "c2u": (1 << 27, 1 << 29, 0.0, (4, 4, 1), "plain equi-join |R|=2^27 |S|=2^29 uniform, groups of 4"),
    "c2z": (1 << 27, 1 << 29, 1.5, (4, 4, 1), "plain equi-join |R|=2^27 |S|=2^29 Zipf 1.5, groups of 4"),
    "c3u": (1 << 26, 1 << 29, 0.0, (4, 4, 1), "plain equi-join |R|=2^26 |S|=2^29 uniform, groups of 4"),
    # 1/8 of C2 (same Zipf and layout): the small case for ncu captures
    "c2s": (1 << 24, 1 << 26, 1.0, (4, 4, 1), "plain equi-join |R|=2^24 |S|=2^26 Zipf 1.0, groups of 4"),
}
SEED = 0x5EED5EED
METRIC = "join tuples/s (|R|+|S|)"


def launches_per_join(alg, radix_bits, single=True, heavy=False):
    """Kernels of this library one plan execution launches (see launch_pipeline):
    k_init_single for a single-join plan; the non-partitioned join has no
    partitioning passes; a second scatter pass (and its work list) above 8 radix
    bits; the heavy-key sample and the heavy first scatter pass when the plan
    samples heavy keys."""
    n = 1 if single else 0
    if alg == 1:
        return n + 8
    return n + 10 + (2 if radix_bits > 8 else 0) + (2 if heavy else 0)


def samples_heavy(args, n_s, alg=None):
    """Whether the plan samples heavy keys for this join (the planner's rule)."""
    if args.alg == 1 or alg == 1 or args.heavy < 0:
        return False
    return args.heavy > 0 or (args.skew == 0 and n_s >= (1 << 24))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return ws, int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def emit(obj):
    print(json.dumps(obj), flush=True)


# ------------------------------------------------------------ CPU baseline --
def _oracle():
    """The oracle (test infrastructure): the CPU arms' only library. They load
    no product library, so nothing of this repository's GPU path runs there."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def cpu_reference_run(n_r, n_s, zipf, layout, steps, warmup, data=None):
    """The reference's pipeline restated in C (the oracle's port of its global
    partition, rank-set / bank-set replication and local hash join) on all host
    cores, over the whole workload: `warmup` untimed and `steps` timed joins.
    `data` = (R, S, expected checksum) as host arrays, else the oracle's own copy
    of the seeded generator makes them. Returns (seconds per timed step, sample
    description, threads)."""
    oracle = _oracle()
    ranks, rsets, bset = layout
    if data is None:
        data = oracle.generate(n_r, n_s, zipf, seed=SEED)
    R, S, expect = data
    cores = os.cpu_count() or 1
    secs = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        out = oracle.refpipe_join(R, S, ranks=ranks, rank_sets=rsets, bank_set=bset, alg=0, nthreads=cores)
        dt = time.perf_counter() - t0
        if i == 0 and (out.shape[0] != n_s or oracle.checksum(out) != expect & (2**64 - 1)):
            raise SystemExit("CPU restatement disagrees with the generator's expected join")
        del out
        if i >= warmup:
            secs.append(dt)
    sample = (f"the whole workload (|R|={n_r}, |S|={n_s}, Zipf {zipf:g}, -r {ranks} -R {rsets} -B {bset}), "
              f"reference pipeline restated in C (oracle), {cores} threads, {steps} timed joins")
    return secs, sample, cores


def cpu_reference_specs(specs, steps, warmup, budget_tuples=24 << 20):
    """The reference pipeline restated in C on all host cores over a mix of
    joins: each step joins the first joins of `specs` whose sizes add up to
    about `budget_tuples` (every join in full), and the rate is their tuples
    over the summed time."""
    oracle = _oracle()
    take, tot = [], 0
    for n_r, n_s, z in specs:
        if tot + n_r + n_s > budget_tuples and take:
            continue
        take.append((n_r, n_s, z))
        tot += n_r + n_s
    data = [oracle.generate(n_r, n_s, z, seed=SEED + 77 + i) for i, (n_r, n_s, z) in enumerate(take)]
    cores = os.cpu_count() or 1
    rates = []
    for it in range(warmup + steps):
        el = 0.0
        for (n_r, n_s, _), (R, S, expect) in zip(take, data):
            t0 = time.perf_counter()
            out = oracle.refpipe_join(R, S, ranks=1, rank_sets=1, bank_set=1, alg=0, nthreads=cores)
            el += time.perf_counter() - t0
            if it == 0:
                assert out.shape[0] == n_s and oracle.checksum(out) == expect, "CPU restatement disagrees"
        if it >= warmup:
            rates.append(tot / el)
    sample = (f"{len(take)} joins of the mix ({tot} tuples, each join in full), reference pipeline restated "
              f"in C, {cores} threads")
    return rates, sample, cores, tot


def run_reference(args):
    """The reference arm: the reference's join algorithm restated in C, on the
    host cores, on the same workload; rank 0 alone under torchrun."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload in ("c4", "c5"):
        specs = c4_specs(scale=args.c4_scale) if args.workload == "c4" else c5_specs(args.c5_pool)
        rates, sample, cores, tot = cpu_reference_specs(specs, args.steps, args.warmup)
        desc = ("batched joins, |R| log-uniform [2^12, 2^24], R:S in {1,2,4,8}, Zipf s ~ U[0, 1.5]"
                if args.workload == "c4" else
                "served join stream, |R| log-uniform [2^10, 2^22], R:S in {1,2,4,8}, Zipf s ~ U[0, 1.5]")
        v = statistics.median(rates)
        ms_step = tot / v * 1e3
    else:
        n_r, n_s, zipf, layout, desc = workload_spec(args)
        secs, sample, cores = cpu_reference_run(n_r, n_s, zipf, layout, args.steps, args.warmup)
        ms_step = statistics.mean(secs) * 1e3
        v = (n_r + n_s) / (ms_step / 1e3)
    emit({"impl": "reference", "metric": METRIC, "value": v, "unit": "tuples/s", "n_gpus": args.gpus,
          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
          "config": {"workload": desc, "sample": sample},
          "cpu_baseline": {"value": v, "unit": "tuples/s", "cores": cores, "kind": "port", "sample": sample},
          "e2e": {"value": v, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return 0


def workload_spec(args):
    """The workload's sizes, skew, rank layout (-r, -R, -B) and description;
    --groups G replaces the layout by G rank sets of one rank each (-r G -R G -B 1)."""
    n_r, n_s, zipf, layout, desc = WORKLOADS[args.workload]
    if args.groups > 0:
        g = args.groups
        layout = (g, g, 1)
        desc = (desc.split(", groups of")[0].split(", replication groups of")[0] +
                f", replication groups of {g} (-r {g} -R {g} -B 1)")
    return n_r, n_s, zipf, layout, desc


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid=None, period_ms=20):
        """Starts nvidia-smi sampling every `period_ms` and waits (at most 5 s)
        for its first sample, so that sampling is running before the timed
        region begins."""
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", str(period_ms)]
        if uuid:
            cmd.append("--id=" + uuid)
        self.mark_rows = 0
        try:
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 5.0 and not self._rows():
            time.sleep(0.02)

    def _rows(self):
        self.f.flush()
        with open(self.f.name) as g:
            return [ln.strip().split(", ") for ln in g if ln.strip()]

    def mark(self):
        """The timed region starts now: only later samples are reported."""
        if self.p is not None:
            self.mark_rows = len(self._rows())

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        rows = self._rows()
        os.unlink(self.f.name)
        timed = rows[self.mark_rows:]
        # a timed region shorter than the sampling period: the last sample before its end
        rows, window = (timed, "timed region") if timed else (rows[-1:], "last sample before the timed region ended")
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for name, val in zip(names, r[5:9]):
                    if val.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "window": window}


# ---------------------------------------------------------------- our arm --
def traffic_from_profiles(kernel, units):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, scaled
    to `units` tuples when the capture used a smaller case."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            t = json.load(f)
        k = t["kernels"][kernel]
        return k["dram_bytes"] * units / k["units"]
    except Exception:
        return None


def device_join_leg(spj, n_r, n_s, zipf, layout, args, steps, warmup, seed, sample_clocks, keep_inputs=False):
    """One plain join of the given shape with R and S resident in HBM (seeded,
    generated on the device): `warmup` untimed steps and a result check (count
    and checksum against the generator's exact answer), then `steps` steps
    bracketed by CUDA events on the launching stream, with the SM clocks sampled
    inside the timed region. Returns a dict; with keep_inputs it holds the
    device columns for the end-to-end leg."""
    import torch
    ranks, rsets, bset = layout
    design = spj.make_design(rank_num=ranks, rank_set=rsets, bank_set=bset, join_alg=args.alg,
                             skew_mode=args.skew, input_size=n_r, rs_ratio=max(n_s // n_r, 1),
                             zipf_factor=int(round(zipf * 100)), radix_bits=args.bits,
                             table_slots=args.slots, unit_tuples=args.unit, heavy_sample=args.heavy)
    ws, rank, local = dist_env()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    lib = spj.lib()
    dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
    dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
    expect = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(lib.spj_generate_device(seed, n_r, n_s, zipf, dR.data_ptr(), dS.data_ptr(), expect.data_ptr(), sp))
    plan = spj.Plan(n_r, n_s, design)
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    csum = torch.zeros(1, dtype=torch.int64, device="cuda")

    def step():
        plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n_out.data_ptr(), sp)

    for _ in range(warmup):
        step()
    spj.check(lib.spj_checksum_device(out.data_ptr(), n_out.data_ptr(), csum.data_ptr(), sp))
    torch.cuda.synchronize()
    st = plan.stats()
    ok = int(n_out.item()) == n_s and int(csum.item()) == int(expect.item())
    if not ok:
        raise SystemExit(f"join result check failed: {int(n_out.item())} pairs, checksum mismatch")
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid) if sample_clocks else None
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if sampler:
        sampler.mark()
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1)
    kts = [plan.kernel_times(b) for b in range(min(steps, 128))]
    kmean = {k: statistics.mean(x[k] for x in kts) for k in kts[0]}
    res = {"ms": ms, "ms_step": ms / steps, "kmean": kmean, "stats": st, "n_pairs": int(n_out.item()),
           "ok": ok, "clocks": clocks, "design": design, "expect": int(expect.item())}
    del out
    plan.close()
    if keep_inputs:
        res["dR"], res["dS"] = dR, dS
    else:
        del dR, dS
    torch.cuda.empty_cache()
    return res


def run_ours(args):
    import torch
    import spidjoin as spj

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n_r, n_s, zipf, (ranks, rsets, bset), desc = workload_spec(args)
    if dist:  # every rank warmed up and checked before the common timed region
        dist.barrier()
    leg = device_join_leg(spj, n_r, n_s, zipf, (ranks, rsets, bset), args, args.steps, args.warmup, SEED + rank,
                          rank == 0, keep_inputs=True)
    ms = leg["ms"]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = ws * (n_r + n_s) / (ms_step / 1e3)
    kmean, st, n_pairs, design = leg["kmean"], leg["stats"], leg["n_pairs"], leg["design"]
    dR, dS = leg.pop("dR"), leg.pop("dS")
    alg_bytes = {  # algorithmic bytes per launch
        "k_hist": 8 * (n_r + n_s),
        "k_scatter": 16 * (n_r + n_s),
        "k_join_phj": 8 * (n_r + n_s) + 8 * n_pairs,
    }
    times = {"k_hist": kmean["hist_ms"], "k_scatter": kmean["scatter_ms"], "k_join_phj": kmean["join_ms"]}
    if st["join_alg"] == 1:  # non-partitioned: the table's clear and build, then the probe over S
        alg_bytes = {"k_nphj_build": 16 * n_r, "k_nphj_probe": 8 * n_s + 8 * n_pairs}
        times = {"k_nphj_build": kmean["scatter_ms"], "k_nphj_probe": kmean["join_ms"]}
    dom = max(times, key=times.get)
    peak, peak_kind = peaks()
    achieved = alg_bytes[dom] / (times[dom] / 1e3) / 1e9
    traffic = traffic_from_profiles(dom, n_r + n_s)
    pipe_bytes = 24 * (n_r + n_s) + 8 * n_pairs
    pipe_gbs = pipe_bytes / (ms_step / 1e3) / 1e9

    # end to end through the JoinInstance API with pinned host columns
    e2e = None
    hR = hS = None
    if not args.no_e2e or (rank == 0 and ws == 1 and not args.no_cpu):
        hR = torch.empty((n_r, 2), dtype=torch.int32, pin_memory=True)
        hS = torch.empty((n_s, 2), dtype=torch.int32, pin_memory=True)
        hR.copy_(dR)
        hS.copy_(dS)
    del dR, dS
    torch.cuda.empty_cache()
    if not args.no_e2e:
        inst = spj.JoinInstance(ranks, rsets, ranks // rsets)
        inst.LoadColumn((hR.data_ptr(), n_r), n_r, "left")
        inst.LoadColumn((hS.data_ptr(), n_s), n_s, "right")
        inst.PrepareJoin(design)
        ke = max(2, min(args.steps, 5))
        for _ in range(1):
            inst.StartJoin(design)
            inst.FinishJoin(copy=False)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        got = 0
        for _ in range(ke):
            inst.StartJoin(design)
            res = inst.FinishJoin(copy=False)
            got = sum(res.byte_sizes) // 8
        el = time.perf_counter() - t0
        if dist:
            t = torch.tensor([el], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        inst.close()
        e2e = {"value": ws * (n_r + n_s) * ke / el, "unit": "tuples/s", "steps": ke,
               "h2d_bytes_per_step": 8 * (n_r + n_s), "d2h_bytes_per_step": 8 * got + 8,
               "ms_per_step": el / ke * 1e3}

    # the CPU baseline: the reference pipeline restated in C on the same bytes
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        import numpy as np
        R = hR.numpy().view(np.uint32)
        S = hS.numpy().view(np.uint32)
        secs, sample, cores = cpu_reference_run(n_r, n_s, zipf, (ranks, rsets, bset), 1, 1,
                                                data=(R, S, leg["expect"]))
        cpu = {"value": (n_r + n_s) / statistics.mean(secs), "unit": "tuples/s", "cores": cores, "kind": "port",
               "sample": sample, "ms_per_step": statistics.mean(secs) * 1e3}
        del R, S
    del hR, hS

    # the target comparisons on the same GPU: the C2 shape at Zipf 1.5
    # against uniform, the batched form of config 4 against one plain join per
    # join (every join checked), and config 3's sort-merge against its hash join
    extra = {}
    if rank == 0 and ws == 1 and args.workload == "c2" and not args.no_extra:
        k = max(3, min(args.steps, 10))
        uni = device_join_leg(spj, n_r, n_s, 0.0, (ranks, rsets, bset), args, k, 3, SEED + 11, True)
        z15 = device_join_leg(spj, n_r, n_s, 1.5, (ranks, rsets, bset), args, k, 3, SEED + 12, True)
        extra["skew"] = {
            "workload": f"|R|=2^27 |S|=2^29, -r {ranks} -R {rsets} -B {bset}: uniform vs Zipf 1.5",
            "uniform_ms": uni["ms_step"], "zipf_1_5_ms": z15["ms_step"], "zipf_1_0_ms": ms_step,
            "zipf_1_5_vs_uniform": z15["ms_step"] / uni["ms_step"], "target": "<= 1.5",
            "steps": k, "checked": uni["ok"] and z15["ok"],
            "kernels_ms": {"uniform": uni["kmean"], "zipf_1_5": z15["kmean"]},
            "heavy_keys": {"uniform": uni["stats"]["heavy_keys"], "zipf_1_5": z15["stats"]["heavy_keys"]},
            "clocks": {"uniform": uni["clocks"], "zipf_1_5": z15["clocks"]}}
        extra["batched"] = batched_compare(spj, args, steps=max(3, min(args.steps, 5)), warmup=3)
        # config 3 with the sort-merge local join against the hash join (both checked)
        import copy
        n3r, n3s, z3, lay3, _ = WORKLOADS["c3"]
        legs = {}
        for name, alg in (("hash", 0), ("sort_merge", 2)):
            a = copy.copy(args)
            a.alg = alg
            legs[name] = device_join_leg(spj, n3r, n3s, z3, lay3, a, k, 3, SEED + 13, True)
        # config 1, the reference driver's own case (-s 1048576 -t 2), as the planner runs it
        n1r, n1s, z1, lay1, _ = WORKLOADS["c1"]
        c1 = device_join_leg(spj, n1r, n1s, z1, lay1, args, max(20, args.steps), 5, SEED + 14, True)
        b1 = 24 * (n1r + n1s) + 8 * c1["n_pairs"]
        extra["c1"] = {"workload": WORKLOADS["c1"][4], "ms_per_step": c1["ms_step"],
                       "value": (n1r + n1s) / (c1["ms_step"] / 1e3), "unit": "tuples/s", "checked": c1["ok"],
                       "join_alg_run": c1["stats"]["join_alg"],
                       "pipeline_roofline": {"frac": b1 / (c1["ms_step"] / 1e3) / 1e9 / peak, "peak": peak},
                       "kernels_ms": c1["kmean"], "clocks": c1["clocks"]}
        extra["sort_merge"] = {
            "workload": f"|R|=2^26 |S|=2^29 Zipf {z3:g}, -r {lay3[0]} -R {lay3[1]} -B {lay3[2]}: sort-merge vs hash join",
            "hash_ms": legs["hash"]["ms_step"], "sort_merge_ms": legs["sort_merge"]["ms_step"],
            "sort_merge_vs_hash": legs["sort_merge"]["ms_step"] / legs["hash"]["ms_step"], "target": "<= 1.3",
            "steps": k, "checked": legs["hash"]["ok"] and legs["sort_merge"]["ok"],
            "join_alg_run": {n: legs[n]["stats"]["join_alg"] for n in legs},
            "kernels_ms": {n: legs[n]["kmean"] for n in legs}, "clocks": {n: legs[n]["clocks"] for n in legs}}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": desc, "n_r": n_r, "n_s": n_s, "zipf": zipf, "rank_num": ranks,
                       "rank_set": rsets, "bank_set": bset, "join_alg": args.alg, "join_alg_run": st["join_alg"],
                       "skew_mode": "adaptive" if args.skew == 0 else "fixed",
                       "radix_bits": st["radix_bits"], "table_slots": st["table_slots"],
                       "l2": "inputs (8*(|R|+|S|) bytes) larger than the 126 MB L2; no flush",
                       "seed": SEED, "parallelism": f"replicas x{ws}"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg_bytes[dom], "traffic": traffic},
            "pipeline_roofline": {"achieved": pipe_gbs, "peak": peak, "unit": "GB/s", "frac": pipe_gbs / peak,
                                  "algorithmic_bytes": pipe_bytes, "formula": "24*(|R|+|S|) + 8*|out|"},
            "kernels_ms": kmean,
            "e2e": e2e, "cpu_baseline": cpu,
            "gpu_launches": launches_per_join(st["join_alg"], st["radix_bits"], heavy=samples_heavy(args, n_s, st["join_alg"])) * args.steps,
            "clocks": leg["clocks"],
            "check": {"n_pairs": n_pairs, "checksum_ok": leg["ok"], "max_s_partition": st["max_s_partition"],
                      "units": st["units"], "heavy_keys": st["heavy_keys"], "heavy_tuples": st["heavy_tuples"]},
        }
        line.update(extra)
        emit(line)
    if dist:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------- sharded (N > 1) --
def run_distributed(args):
    """One join over N GPUs: every rank holds a shard of R and of S (the
    workload's sizes per rank: weak scaling; rank i's keys are its generator's
    keys + i*|R|, so the global R has unique keys), splits both by destination
    rank, exchanges them with NCCL all-to-all and joins what it received. The
    timed step is the whole distributed join; time = max over ranks."""
    import datetime
    import torch
    import torch.distributed as dist
    import spidjoin as spj

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if "MASTER_ADDR" not in os.environ:  # one process without torchrun (--sharded)
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]), RANK="0",
                              WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    n_r, n_s, zipf, (ranks, rsets, bset), desc = workload_spec(args)
    design = spj.make_design(rank_num=ranks, rank_set=rsets, bank_set=bset, join_alg=args.alg,
                             skew_mode=args.skew, input_size=n_r, rs_ratio=max(n_s // n_r, 1),
                             zipf_factor=int(round(zipf * 100)), radix_bits=args.bits,
                             table_slots=args.slots, unit_tuples=args.unit)
    lib = spj.lib()
    stream = torch.cuda.current_stream()
    dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
    dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
    expect = torch.zeros(1, dtype=torch.int64, device="cuda")
    spj.check(lib.spj_generate_device(SEED + rank, n_r, n_s, zipf, dR.data_ptr(), dS.data_ptr(),
                                      expect.data_ptr(), stream.cuda_stream))
    dR[:, 0] += rank * n_r
    dS[:, 0] += rank * n_r
    csum = torch.zeros(1, dtype=torch.int64, device="cuda")

    def checked_warmup(dj):
        """Warm-up steps, then the all-reduced checksum and count; every rank
        gets the same verdict. A failing setup counts as a wrong result."""
        ok = torch.ones(1, dtype=torch.int64, device="cuda")
        try:
            for _ in range(args.warmup):
                pairs, n = dj.run(dR, dS)
            spj.check(lib.spj_checksum_device(pairs.data_ptr(), n.data_ptr(), csum.data_ptr(), stream.cuda_stream))
            tot = torch.stack([csum[0], expect[0], n[0]])
        except Exception as exc:  # noqa: BLE001 -- reported and replaced by the all-to-all exchange
            print(f"rank {rank}: exchange setup failed: {exc}", file=sys.stderr)
            ok.zero_()
            tot = torch.zeros(3, dtype=torch.int64, device="cuda")
        dist.all_reduce(ok, op=dist.ReduceOp.MIN)
        dist.all_reduce(tot)
        return bool(ok.item()) and int(tot[0].item()) == int(tot[1].item()) and int(tot[2].item()) == ws * n_s

    # the split fused into the send (peer stores into symmetric memory) first;
    # the NCCL all-to-all exchange if that cannot be set up or checks wrong
    exchange = "fused split-and-send into peer receive buffers (symmetric memory, NVLink)"
    dj = spj.DistributedJoin(design=design, fused=args.exchange == "fused")
    if not checked_warmup(dj):
        if args.exchange != "fused":
            raise SystemExit("distributed join result check failed")
        dj.close()
        exchange = "NCCL all-to-all (the fused exchange failed its check)"
        dj = spj.DistributedJoin(design=design)
        if not checked_warmup(dj):
            raise SystemExit("distributed join result check failed")
    if args.exchange != "fused":
        exchange = "device split, NCCL all-to-all"
    sampler = ClockSampler() if rank == 0 else None
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.mark()
    ev0.record(stream)
    for _ in range(args.steps):
        pairs, n = dj.run(dR, dS)
    ev1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop() if sampler else None
    t = torch.tensor([ev0.elapsed_time(ev1) / args.steps], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item())
    local_out = torch.tensor([float(n.item())], dtype=torch.float64, device="cuda")
    dist.all_reduce(local_out, op=dist.ReduceOp.MAX)
    del pairs
    # end to end: shards from pinned host memory, the distributed join, pairs back to pinned host memory
    e2e = None
    if not args.no_e2e:
        hR = torch.empty((n_r, 2), dtype=torch.int32, pin_memory=True)
        hS = torch.empty((n_s, 2), dtype=torch.int32, pin_memory=True)
        hR.copy_(dR)
        hS.copy_(dS)
        hout = torch.empty((int(local_out.item()) + (1 << 20), 2), dtype=torch.int32, pin_memory=True)
        ke, got, el = 2, 0, 0.0
        for i in range(ke + 1):
            dist.barrier()
            t0 = time.perf_counter()
            dR.copy_(hR, non_blocking=True)
            dS.copy_(hS, non_blocking=True)
            pairs, n = dj.run(dR, dS)
            k = int(n.item())
            if k > hout.shape[0]:
                hout = torch.empty((k, 2), dtype=torch.int32, pin_memory=True)
            hout[:k].copy_(pairs[:k], non_blocking=True)
            torch.cuda.synchronize()
            if i > 0:
                el += time.perf_counter() - t0
                got += k
            del pairs
        te = torch.tensor([el], dtype=torch.float64, device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": ws * (n_r + n_s) * ke / float(te.item()), "unit": "tuples/s", "steps": ke,
               "h2d_bytes_per_step": 8 * (n_r + n_s), "d2h_bytes_per_step": 8 * got // ke,
               "ms_per_step": float(te.item()) / ke * 1e3, "per": "rank 0's copies; time max over ranks"}
        del hR, hS, hout
    dj.close()
    peak, peak_kind = peaks()
    pipe_bytes = ws * (24 * (n_r + n_s) + 8 * n_s)
    if rank == 0:
        emit({
            "metric": METRIC, "value": ws * (n_r + n_s) / (ms_step / 1e3), "unit": "tuples/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": desc + f"; per rank, sharded over {ws} GPUs (rank i keys + i*|R|)",
                       "exchange": exchange,
                       "n_r_per_rank": n_r, "n_s_per_rank": n_s, "zipf": zipf, "join_alg": args.alg,
                       "parallelism": f"hash exchange over {ws} ranks, local joins",
                       "l2": "inputs larger than L2; no flush", "seed": SEED},
            "pipeline_roofline": {"achieved": pipe_bytes / ws / (ms_step / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                  "frac": pipe_bytes / ws / (ms_step / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                                  "formula": "per rank: 24*(|R|+|S|) + 8*|out|, exchange not counted"},
            "max_local_pairs": local_out.item(),
            "e2e": e2e, "cpu_baseline": None, "gpu_launches": (6 + launches_per_join(args.alg, 15)) * args.steps,
            "clocks": clocks,
            "check": {"global_checksum_ok": True, "pairs": ws * n_s},
        })
    dist.destroy_process_group()
    return 0


# ----------------------------------------------------------- batched (c4) --
def c4_specs(n_joins=256, seed=SEED + 4, scale=1.0):
    """Config 4: |R| log-uniform in [2^12, 2^24], R:S ratio from {1,2,4,8}, Zipf s
    uniform in [0, 1.5], all from one seed (numpy's PCG64)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_joins):
        n_r = max(1, int(2.0 ** rng.uniform(12.0, 24.0) * scale))
        ratio = int(rng.choice([1, 2, 4, 8]))
        specs.append((n_r, n_r * ratio, float(rng.uniform(0.0, 1.5))))
    return specs


def batched_compare(spj, args, steps, warmup):
    """Config 4: the 256 joins as one batch plan replayed from a CUDA graph,
    against one pre-created plain plan per join (the device times of its
    executions summed); every join of both forms checked against the
    generator's exact count and checksum. Returns a dict."""
    import torch
    specs = c4_specs(scale=args.c4_scale)
    J = len(specs)
    tot = sum(a + b for a, b, _ in specs)
    lib = spj.lib()
    design = spj.make_design(rank_num=1, join_alg=args.alg, skew_mode=args.skew)
    tuning = None
    if args.tuning and os.path.exists(args.tuning):
        spj.load_tuning(args.tuning)  # the autotuner's per-class table (spid-join_b200/autotune.py)
        tuning = os.path.relpath(args.tuning, ROOT)
    R, S, exp = [], [], []
    for i, (n_r, n_s, z) in enumerate(specs):
        dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
        dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
        e = torch.zeros(1, dtype=torch.int64, device="cuda")
        spj.check(lib.spj_generate_device(SEED + 1000 + i, n_r, n_s, z, dR.data_ptr(), dS.data_ptr(), e.data_ptr(),
                                          None))
        R.append(dR)
        S.append(dS)
        exp.append(e)
    torch.cuda.synchronize()
    exp_t = torch.cat(exp)
    n_s_t = torch.tensor([b for _, b, _ in specs], dtype=torch.int64, device="cuda")

    def wrong(outs, n_out):
        """Joins whose count or checksum differs from the generator's answer."""
        cs = torch.zeros(J, dtype=torch.int64, device="cuda")
        for j in range(J):
            spj.check(lib.spj_checksum_device(outs[j].data_ptr(), n_out[j:j + 1].data_ptr(), cs[j:j + 1].data_ptr(),
                                              None))
        torch.cuda.synchronize()
        return int(((cs != exp_t) | (n_out != n_s_t)).sum().item())

    batch = spj.Batch([a for a, _, _ in specs], [b for _, b, _ in specs], design)
    outs = [torch.empty((batch.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(J)]
    n_out = torch.zeros(J, dtype=torch.int64, device="cuda")
    batch.bind([t.data_ptr() for t in R], [t.data_ptr() for t in S], [o.data_ptr() for o in outs], n_out.data_ptr())
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        batch.execute(side.cuda_stream)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batch.execute(torch.cuda.current_stream().cuda_stream)
    for _ in range(warmup):
        graph.replay()
    torch.cuda.synchronize()
    bad = wrong(outs, n_out)
    if bad:
        raise SystemExit(f"batched join check failed for {bad} joins")
    sampler = ClockSampler()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    sampler.mark()
    ev0.record()
    for _ in range(steps):
        graph.replay()
    ev1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms_batched = ev0.elapsed_time(ev1) / steps
    del graph
    batch.execute(0)  # one eager run for the per-kernel split
    kmean = batch.kernel_times(0)
    batch.close()

    # plain: one plan per join, its device time per execution, summed over joins
    plain_ms = 0.0
    n_out.zero_()
    plain_outs = []
    for j, (n_r, n_s, z) in enumerate(specs):
        plan = spj.Plan(n_r, n_s, design)
        o = outs[j] if outs[j].shape[0] >= plan.output_capacity else \
            torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
        plain_outs.append(o)
        n1 = n_out[j:j + 1]
        plan.execute(R[j].data_ptr(), S[j].data_ptr(), o.data_ptr(), n1.data_ptr(), 0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        a.record()
        for _ in range(reps):
            plan.execute(R[j].data_ptr(), S[j].data_ptr(), o.data_ptr(), n1.data_ptr(), 0)
        b.record()
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(b) / reps
        plan.close()
    bad = wrong(plain_outs, n_out)
    if bad:
        raise SystemExit(f"plain join check failed for {bad} joins")

    # plain, back to back: every join's plan created first, then the J executions
    # on one stream between two events, so the gaps between the joins count too
    seq = {"how": "one pre-created plan per join, the J executions back to back on one stream, CUDA events "
                  "around the sequence"}
    plans = []
    try:
        for n_r, n_s, _ in specs:
            plans.append(spj.Plan(n_r, n_s, design))
        souts = [outs[j] if outs[j].shape[0] >= plans[j].output_capacity else plain_outs[j] for j in range(J)]

        def run_all():
            for j in range(J):
                plans[j].execute(R[j].data_ptr(), S[j].data_ptr(), souts[j].data_ptr(), n_out[j:j + 1].data_ptr(), 0)

        n_out.zero_()
        run_all()
        torch.cuda.synchronize()
        bad = wrong(souts, n_out)
        if bad:
            raise SystemExit(f"plain back-to-back check failed for {bad} joins")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        a.record()
        for _ in range(reps):
            run_all()
        b.record()
        torch.cuda.synchronize()
        seq_ms = a.elapsed_time(b) / reps
        seq.update({"value": tot / (seq_ms / 1e3), "ms_per_step": seq_ms, "batched_vs_this": seq_ms / ms_batched})
    except spj.SpjError as e:  # the plans of all joins at once may not fit
        seq["skipped"] = str(e)
    finally:
        for pl in plans:
            pl.close()
    pipe_bytes = sum(24 * (a + b) + 8 * b for a, b, _ in specs)
    peak, peak_kind = peaks()
    del outs, plain_outs, R, S
    torch.cuda.empty_cache()
    return {"workload": f"batched: {J} joins, |R| log-uniform [2^12, 2^24], R:S in {{1,2,4,8}}, "
                        f"Zipf s ~ U[0, 1.5], one seed; one CUDA graph per step",
            "joins": J, "tuples": tot, "scale": args.c4_scale, "tuning": tuning,
            "value": tot / (ms_batched / 1e3), "ms_per_step": ms_batched, "steps": steps,
            "plain": {"value": tot / (plain_ms / 1e3), "ms_per_step": plain_ms,
                      "how": "one pre-created plan per join, CUDA-event device time per execution, summed"},
            "plain_back_to_back": seq,
            "batched_vs_plain": plain_ms / ms_batched, "target": ">= 3",
            "pipeline_roofline": {"achieved": pipe_bytes / (ms_batched / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                  "frac": pipe_bytes / (ms_batched / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
            "clocks": clocks, "kernels_ms_eager": kmean,
            "check": {"joins_checked": 2 * J, "all_exact": True,
                      "how": "count and 64-bit checksum of every join, batched and plain"}}


def run_batched(args):
    import torch
    import spidjoin as spj

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    r = batched_compare(spj, args, args.steps, args.warmup)
    emit({
        "metric": METRIC, "value": r["value"], "unit": "tuples/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": r["workload"], "joins": r["joins"], "tuples": r["tuples"], "join_alg": args.alg,
                   "scale": args.c4_scale, "tuning": r["tuning"], "l2": "inputs larger than L2; no flush"},
        "plain": r["plain"], "batched_vs_plain": r["batched_vs_plain"],
        "pipeline_roofline": r["pipeline_roofline"],
        "gpu_launches": launches_per_join(args.alg, 15, single=False) * args.steps, "clocks": r["clocks"],
        "kernels_ms_eager": r["kernels_ms_eager"], "check": r["check"],
    })
    return 0


# ------------------------------------------------------------ served (c5) --
def c5_specs(n_joins, seed=SEED + 5):
    """Config 5's join mix: |R| log-uniform in [2^10, 2^22], R:S ratio from
    {1,2,4,8}, Zipf s uniform in [0, 1.5] (numpy's PCG64)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_joins):
        n_r = int(2.0 ** rng.uniform(10.0, 22.0))
        ratio = int(rng.choice([1, 2, 4, 8]))
        specs.append((n_r, n_r * ratio, float(rng.uniform(0.0, 1.5))))
    return specs


def serve_stream(spj, server, pool, R, S, outs, n_out, rate, seconds, max_outstanding, seed):
    """Drives `server` with joins drawn round-robin from the pool: Poisson
    arrivals at `rate` joins/s for `seconds` (rate = 0: closed loop with
    `max_outstanding` requests in flight). A side-stream checksum and count of
    every output are kept on the device for checking after the run. Returns a
    dict of measurements."""
    import threading
    import numpy as np
    import torch
    P = len(pool)
    lib = spj.lib()
    rng = np.random.default_rng(seed)
    cap_req = int((rate * 1.5 if rate > 0 else 50000) * seconds) + 16
    sums = torch.zeros(cap_req, dtype=torch.int64, device="cuda")
    counts = torch.full((cap_req,), -1, dtype=torch.int64, device="cuda")
    side = torch.cuda.Stream()
    free = [threading.Semaphore(1) for _ in range(P)]  # pool entry p: its output is not in use
    checked = [torch.cuda.Event() for _ in range(P)]  # the side-stream check of entry p's last output
    outstanding = threading.Semaphore(max_outstanding)
    queue, qcv = [], threading.Condition(threading.Lock())
    done_flag = [False]
    lat, entries, late = [], [], []
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=cap_req)) if rate > 0 else None

    def waiter():
        k = 0
        while True:
            with qcv:
                while k >= len(queue) and not done_flag[0]:
                    qcv.wait(0.05)
                if k >= len(queue):
                    return
                rid, p = queue[k]
            lat.append(server.wait(rid, -1.0))
            with torch.cuda.stream(side):
                counts[k:k + 1].copy_(n_out[p:p + 1])
                spj.check(lib.spj_checksum_device(outs[p].data_ptr(), n_out[p:p + 1].data_ptr(),
                                                  sums[k:k + 1].data_ptr(), side.cuda_stream))
                checked[p].record(side)
            free[p].release()
            outstanding.release()
            k += 1

    old_switch = sys.getswitchinterval()
    sys.setswitchinterval(0.0002)
    w = threading.Thread(target=waiter)
    w.start()
    t0 = time.perf_counter()
    k = 0
    while k < cap_req:
        now = time.perf_counter() - t0
        if now >= seconds:
            break
        if arrivals is not None and arrivals[k] > now:
            time.sleep(arrivals[k] - now)
            continue
        p = k % P
        outstanding.acquire()
        free[p].acquire()
        checked[p].synchronize()
        if arrivals is not None:
            late.append(time.perf_counter() - t0 - arrivals[k])
        n_r, n_s, _ = pool[p]
        rid = server.submit(R[p].data_ptr(), n_r, S[p].data_ptr(), n_s, outs[p].data_ptr(), outs[p].shape[0],
                            n_out[p:p + 1].data_ptr())
        with qcv:
            queue.append((rid, p))
            qcv.notify()
        entries.append(p)
        k += 1
    with qcv:
        done_flag[0] = True
        qcv.notify()
    w.join()
    elapsed = time.perf_counter() - t0
    torch.cuda.synchronize()
    sys.setswitchinterval(old_switch)
    n = len(entries)
    return {"requests": n, "elapsed_s": elapsed, "latencies_ms": lat, "entries": entries,
            "sums": sums[:n], "counts": counts[:n], "late_s": late,
            "tuples": sum(pool[p][0] + pool[p][1] for p in entries)}


def run_served(args):
    import numpy as np
    import torch
    import spidjoin as spj

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    lib = spj.lib()
    P = args.c5_pool
    pool = c5_specs(P)
    design = spj.make_design(rank_num=1, join_alg=args.alg, skew_mode=args.skew)
    budget = 120 << 30
    server = spj.Server(hbm_budget_bytes=budget, max_batch=args.c5_max_batch, streams=args.c5_streams,
                        design=design)
    R, S, outs, exp = [], [], [], []
    for i, (n_r, n_s, z) in enumerate(pool):
        dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
        dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
        e = torch.zeros(1, dtype=torch.int64, device="cuda")
        spj.check(lib.spj_generate_device(SEED + 5000 + i, n_r, n_s, z, dR.data_ptr(), dS.data_ptr(), e.data_ptr(),
                                          None))
        R.append(dR)
        S.append(dS)
        exp.append(e)
        outs.append(torch.empty((server.output_capacity(n_r, n_s), 2), dtype=torch.int32, device="cuda"))
    n_out = torch.zeros(P, dtype=torch.int64, device="cuda")
    exp = torch.cat(exp)
    n_s_t = torch.tensor([b for _, b, _ in pool], dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()

    def wrong(run):
        idx = torch.tensor(run["entries"], dtype=torch.int64, device="cuda")
        return int(((run["sums"] != exp[idx]) | (run["counts"] != n_s_t[idx])).sum().item())

    def summary(run, st):
        lat = np.array(run["latencies_ms"])
        return {"requests": run["requests"], "tuples_per_s": run["tuples"] / run["elapsed_s"],
                "joins_per_s": run["requests"] / run["elapsed_s"], "elapsed_s": run["elapsed_s"],
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(lat.max()), "batches": st["batches"], "mean_batch": st["mean_batch"],
                "max_inflight_batches": st["max_inflight_batches"], "hbm_peak_gib": st["hbm_peak_bytes"] / 2**30,
                "arrival_lag_p99_ms": float(np.percentile(run["late_s"], 99) * 1e3) if run["late_s"] else None,
                "wrong_outputs": wrong(run)}

    def leg(srv, rate, seconds, outstanding, seed):
        srv.reset_stats()
        run = serve_stream(spj, srv, pool, R, S, outs, n_out, rate, seconds, outstanding, seed)
        return summary(run, srv.stats())

    serve_stream(spj, server, pool, R, S, outs, n_out, 0, 1.0, 64, SEED)  # warm-up burst
    sampler = ClockSampler()
    sampler.mark()
    served = leg(server, args.c5_rate, args.c5_seconds, 1 << 20, SEED + 1)
    clocks = sampler.stop()
    sat = leg(server, 0, args.c5_sat_seconds, 256, SEED + 2)
    server.close()
    # the plain per-request join: the same stream served one join at a time
    plain_srv = spj.Server(hbm_budget_bytes=budget, max_batch=1, streams=1, design=design)
    serve_stream(spj, plain_srv, pool, R, S, outs, n_out, 0, 0.5, 8, SEED)
    plain = leg(plain_srv, args.c5_rate, args.c5_plain_seconds, 1 << 20, SEED + 1)
    plain_sat = leg(plain_srv, 0, args.c5_sat_seconds, 256, SEED + 2)
    plain_srv.close()
    bad = served["wrong_outputs"] + sat["wrong_outputs"] + plain["wrong_outputs"] + plain_sat["wrong_outputs"]
    if bad:
        raise SystemExit(f"served join check failed for {bad} outputs")
    emit({
        "metric": METRIC, "value": served["tuples_per_s"], "unit": "tuples/s", "n_gpus": ws,
        "steps": served["requests"], "warmup": 1, "ms_per_step": 1e3 * served["elapsed_s"] / served["requests"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"served join stream: Poisson arrivals at {args.c5_rate:g} joins/s for "
                               f"{args.c5_seconds:g} s; joins drawn round-robin from a pool of {P} with |R| "
                               f"log-uniform [2^10, 2^22], R:S in {{1,2,4,8}}, Zipf s ~ U[0, 1.5]; HBM budget "
                               f"120 GiB", "pool_tuples": sum(a + b for a, b, _ in pool),
                   "max_batch": args.c5_max_batch, "streams": args.c5_streams, "join_alg": args.alg},
        "served": served, "saturated": sat, "plain": plain, "plain_saturated": plain_sat,
        "served_vs_plain_saturated": sat["tuples_per_s"] / plain_sat["tuples_per_s"],
        "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
        "gpu_launches": launches_per_join(args.alg, 15, single=False) * served["batches"], "clocks": clocks,
        "check": {"outputs_checked": served["requests"] + sat["requests"] + plain["requests"] +
                  plain_sat["requests"], "all_exact": True,
                  "how": "count and 64-bit checksum of every output against the generator's"},
    })
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c4", "c5"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--alg", type=int, default=0)
    ap.add_argument("--skew", type=int, default=0, help="0 = adaptive replication, 1 = every partition")
    ap.add_argument("--groups", type=int, default=0, help="replication groups G: -r G -R G -B 1 (0 = the workload's)")
    ap.add_argument("--bits", type=int, default=0, help="radix bits (0 = planner)")
    ap.add_argument("--slots", type=int, default=0, help="table slots per CTA (0 = planner)")
    ap.add_argument("--unit", type=int, default=0, help="max S tuples per work unit (0 = planner)")
    ap.add_argument("--heavy", type=int, default=0,
                    help="S keys sampled for heavy keys joined on the fly (0 = planner, -1 = off)")
    ap.add_argument("--c4-scale", type=float, default=1.0, help="scale of the config-4 relation sizes")
    ap.add_argument("--tuning", default=os.path.join(ROOT, "spid-join_b200", "tuning_b200.json"),
                    help="batched workload: autotuner table to install ('' = the planner alone)")
    ap.add_argument("--c5-rate", type=float, default=2000.0, help="served stream: arrivals per second")
    ap.add_argument("--c5-seconds", type=float, default=60.0, help="served stream: duration")
    ap.add_argument("--c5-plain-seconds", type=float, default=15.0, help="plain per-request stream: duration")
    ap.add_argument("--c5-sat-seconds", type=float, default=8.0, help="closed-loop saturation runs: duration")
    ap.add_argument("--c5-pool", type=int, default=256, help="served stream: distinct joins on the device")
    ap.add_argument("--c5-max-batch", type=int, default=64)
    ap.add_argument("--c5-streams", type=int, default=4)
    ap.add_argument("--replicas", action="store_true", help="N > 1: independent joins instead of one sharded join")
    ap.add_argument("--sharded", action="store_true", help="the sharded join even on one GPU (exchange with itself)")
    ap.add_argument("--exchange", default="fused", choices=["fused", "nccl"], help="sharded join's exchange")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="c2: skip the skew and batched comparisons")
    ap.add_argument("--nr", type=int, default=0, help="custom workload: |R| (with --ns, --zipf)")
    ap.add_argument("--ns", type=int, default=0)
    ap.add_argument("--zipf", type=float, default=0.0)
    args = ap.parse_args()
    if args.nr > 0:
        WORKLOADS["custom"] = (args.nr, args.ns, args.zipf, (1, 1, 1),
                               f"plain equi-join |R|={args.nr} |S|={args.ns} Zipf {args.zipf:g}")
        args.workload = "custom"
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4":
        return run_batched(args)
    if args.workload == "c5":
        return run_served(args)
    if (dist_env()[0] > 1 and not args.replicas) or args.sharded:
        return run_distributed(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
