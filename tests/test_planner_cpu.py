"""The planner on the CPU, through spj_plan_describe: what spj_plan_create
and spj_batch_create would run for a join, computed from the B200's limits
(148 SMs, 227 KiB of shared memory per block) without a device. These are
the rules the kernels and the measurements rely on: when the non-partitioned
join replaces the partitioned one, the fan-out and the pass count, the table
sizes, when heavy keys are sampled, and what the tuning table changes in a
batch."""
import math

import pytest

SMS = 148


def _d(spj, **kw):
    return spj.make_design(**kw)


@pytest.mark.parametrize("n_r", [1, 1000, 1 << 20, (1 << 20) + 1, 1 << 22])
def test_hash_join_alone_up_to_2_22_runs_non_partitioned(spj, n_r):
    sh = spj.describe(n_r, 2 * n_r)
    assert sh["join_alg"] == "nphj" and sh["radix_bits"] == 0 and sh["scatter_passes"] == 0
    # its table: a power of two, at a load of at most 1/4 up to 2^20 R tuples, else 1/2
    g = sh["global_table_slots"]
    assert g & (g - 1) == 0 and g >= 1024
    assert g >= (4 if n_r <= 1 << 20 else 2) * n_r and g < max(2048, 2 * (4 if n_r <= 1 << 20 else 2) * n_r)
    assert sh["heavy_sample"] == 0


@pytest.mark.parametrize("kw", [dict(skew_mode=1), dict(radix_bits=9), dict(join_alg="smj"), dict(join_alg="nl")])
def test_non_partitioned_only_for_the_adaptive_hash_join(spj, kw):
    """Fixed skew mode (the replication knobs shape partitions), an explicit
    fan-out, and the algorithms that keep unmatched S tuples stay partitioned."""
    sh = spj.describe(1 << 20, 1 << 21, _d(spj, **kw))
    assert sh["join_alg"] != "nphj" and sh["radix_bits"] > 0
    if "radix_bits" in kw:
        assert sh["radix_bits"] == kw["radix_bits"]


def test_partitioned_from_2_22_plus_one(spj):
    assert spj.describe((1 << 22) + 1, 1 << 23)["join_alg"] == "phj"


@pytest.mark.parametrize("n_r,n_s,rank_num", [((1 << 22) + 1, 1 << 23, 1), (1 << 26, 1 << 29, 1),
                                              (1 << 27, 1 << 29, 4), (1 << 24, 1 << 24, 64)])
def test_fan_out_rules(spj, n_r, n_s, rank_num):
    """Partitions: the mean R partition at most a third of the table, at least
    64 per rank, at least 8 per SM for a join alone, at most 2^15; a second
    scatter pass beyond 2^8 partitions."""
    sh = spj.describe(n_r, n_s, _d(spj, rank_num=rank_num))
    bits, ts = sh["radix_bits"], sh["table_slots"]
    assert sh["join_alg"] == "phj"
    need = math.ceil(math.log2(max(1, -(-n_r // (12288 // 3)))))
    assert bits == min(max(need, math.ceil(math.log2(8 * SMS)), math.ceil(math.log2(64 * rank_num))), 15)
    assert sh["scatter_passes"] == (2 if bits > 8 else 1)
    assert 1024 <= ts <= 12288 and ts % 2 == 0
    mean = n_r / (1 << bits)
    assert ts >= min(12288, 3 * mean)


def test_config_2_shape(spj):
    """C2 (2^27 x 2^29, -r 4 -R 4): 2^15 partitions in two passes, 12288-slot
    tables, heavy keys sampled, the shape the benchmark line reports."""
    sh = spj.describe(1 << 27, 1 << 29, _d(spj, rank_num=4, rank_set=4))
    assert (sh["join_alg"], sh["radix_bits"], sh["scatter_passes"], sh["table_slots"]) == ("phj", 15, 2, 12288)
    assert sh["heavy_sample"] == 16384 and sh["unit_tuples"] == 65536


def test_sort_merge_tables(spj):
    """Sort-merge: partitions half as large (mean at most a sixth of the
    table) and a table of twice the power of two above the bound on the
    largest partition (its merge sort's two buffers)."""
    sh = spj.describe(1 << 26, 1 << 29, _d(spj, join_alg="smj"))
    bits, ts = sh["radix_bits"], sh["table_slots"]
    mean = (1 << 26) / (1 << bits)
    bound = mean + 6 * math.sqrt(mean) + 32
    assert ts == min(12288, max(1024, 2 * 2 ** math.ceil(math.log2(bound))))
    assert mean <= 12288 / 6


@pytest.mark.parametrize("n_s,heavy,batch,want", [((1 << 24) - 1, 0, 0, 0), (1 << 24, 0, 0, 16384),
                                                  (1 << 24, -1, 0, 0), (1 << 21, 5000, 0, 5000),
                                                  (1 << 20, 0, 1 << 26, 16384), ((1 << 20) - 1, 0, 1 << 26, 0)])
def test_heavy_key_sampling(spj, n_s, heavy, batch, want):
    """Heavy keys are sampled by default from 2^24 S tuples (2^20 in a batch),
    with 16384 keys; heavy_sample > 0 sets the sample, -1 turns it off."""
    n_r = 1 << 23  # a partitioned join alone
    sh = spj.describe(n_r, n_s, _d(spj, heavy_sample=heavy), batch_tuples=batch)
    assert sh["heavy_sample"] == want


def test_batch_members_use_the_tuning_table(spj):
    """In a batch the size class's tuning applies (fan-out offset, table, unit,
    algorithm among those with the same output); a join alone ignores it, and a
    batch member is never swapped for the non-partitioned join by size."""
    saved = spj.get_tuning()
    try:
        spj.set_tuning([])
        base = spj.describe(1 << 16, 1 << 18, batch_tuples=1 << 26)
        assert base["join_alg"] == "phj"
        spj.set_tuning([dict(log2_r=16, log2_ratio=2, radix_bits_delta=1, table_slots=4096, unit_tuples=8192,
                             join_alg=1 + spj.ALG["nphj"])])
        tuned = spj.describe(1 << 16, 1 << 18, batch_tuples=1 << 26)
        assert tuned["join_alg"] == "nphj" and tuned["unit_tuples"] == 8192
        spj.set_tuning([dict(log2_r=16, log2_ratio=2, radix_bits_delta=1, table_slots=4096, unit_tuples=8192,
                             join_alg=0)])
        tuned = spj.describe(1 << 16, 1 << 18, batch_tuples=1 << 26)
        assert tuned["radix_bits"] == base["radix_bits"] + 1 and tuned["table_slots"] == 4096
        # a hash join's class cannot switch it to an algorithm that keeps unmatched S tuples
        spj.set_tuning([dict(log2_r=16, log2_ratio=2, join_alg=1 + spj.ALG["smj"])])
        assert spj.describe(1 << 16, 1 << 18, batch_tuples=1 << 26)["join_alg"] == "phj"
        assert spj.describe(1 << 16, 1 << 18)["join_alg"] == "nphj"  # alone: the size rule, no tuning
    finally:
        spj.set_tuning(saved)


def test_describe_rejects_bad_arguments(spj):
    with pytest.raises(spj.SpjError):
        spj.describe(-1, 10)
    with pytest.raises(spj.SpjError):
        spj.describe(10, 10, num_sms=0)
    with pytest.raises(spj.SpjError):
        spj.describe(10, 10, max_smem_per_block=1024)
    with pytest.raises(spj.SpjError):
        spj.describe(10, 10, _d(spj, rank_num=3, rank_set=2))


def _cli():
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spid-join_b200", "spj_join")
    if not os.path.exists(path):
        pytest.skip("spj_join is not built")
    return path


@pytest.mark.parametrize("args,want", [
    (["-s", "1048576", "-t", "2"], "alg=nphj radix_bits=0 passes=0"),                  # the reference driver's case
    (["-s", "134217728", "-t", "4", "-r", "4", "-R", "4", "-z", "100"],
     "alg=phj radix_bits=15 passes=2 table_slots=12288"),                            # config 2
    (["-s", "67108864", "-t", "8", "-a", "smj"], "alg=smj radix_bits=15 passes=2 table_slots=8192"),
])
def test_cli_explains_without_a_gpu(spj, args, want):
    """spj_join -E prints the plan the reference driver's options give (the
    same planner as the library) and exits 0 without touching a GPU."""
    import subprocess
    out = subprocess.run([_cli(), *args, "-E"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    assert want in out.stdout


def test_cli_explain_rejects_a_bad_design():
    import subprocess
    out = subprocess.run([_cli(), "-s", "100", "-t", "2", "-B", "3", "-E"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 2 and "bank_set" in out.stderr


def test_committed_tuning_table_shapes_batch_members(spj):
    """The tuning table the autotuner wrote for the B200 (tuning_b200.json, which
    bench.py installs for batches) loads, and each entry shapes the plan of a
    batch member of its size class: its fan-out offset against the untuned
    planner, its table, its algorithm. A join alone keeps the planner's own
    shape."""
    import os
    path = os.path.join(os.path.dirname(spj.__file__), "tuning_b200.json")
    saved = spj.get_tuning()
    try:
        spj.set_tuning([])
        table = spj.load_tuning(path)
        assert table["entries"] and spj.get_tuning()
        for e in table["entries"]:
            n_r = 1 << e["log2_r"]
            n_s = n_r << e["log2_ratio"]
            tuned = spj.describe(n_r, n_s, batch_tuples=1 << 26)
            alone_tuned = spj.describe(n_r, n_s)
            spj.set_tuning([])
            plain = spj.describe(n_r, n_s, batch_tuples=1 << 26)
            assert spj.describe(n_r, n_s) == alone_tuned  # a join alone: untouched by the table
            spj.load_tuning(path)
            if e["join_alg"] > 0:
                assert spj.ALG[tuned["join_alg"]] == e["join_alg"] - 1
            if tuned["join_alg"] != "nphj":
                want_bits = min(max(plain["radix_bits"] + e["radix_bits_delta"], 1), 15)
                assert tuned["radix_bits"] == want_bits
                if e["table_slots"] > 0:
                    assert tuned["table_slots"] == min(e["table_slots"], 12288) & ~1
            if e["unit_tuples"] > 0:
                assert tuned["unit_tuples"] == e["unit_tuples"]
    finally:
        spj.set_tuning(saved)
