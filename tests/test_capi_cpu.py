"""CPU tests of the C-ABI library: it loads, exports every symbol the header
declares, keeps the reference's defaults, refuses to run without a GPU, and its
host-side generator produces the specified relations."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "spidjoin.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(spj_[a-z_0-9]+)\s*\(", src)))


def test_exports_every_declared_symbol(spj):
    L = ctypes.CDLL(spj.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(spj.EXPORTS) == set(syms)


def test_design_defaults_follow_reference(spj):
    d = spj.make_design()
    # include/idpHandler.hpp:131-145
    assert (d.input_size, d.rank_num, d.zipf_factor, d.rs_ratio, d.rank_set, d.bank_set, d.join_alg) == \
        (500000, 16, 0, 8, 1, 1, 0)


def test_no_gpu_fails_loudly(spj):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(spj.SpjError, match="NODEVICE"):
        spj.JoinInstance(1, 1, 1)
    with pytest.raises(spj.SpjError, match="NODEVICE"):
        spj.Plan(100, 100)
    with pytest.raises(spj.SpjError, match="NODEVICE"):
        spj.Server(1 << 30)
    with pytest.raises(spj.SpjError, match="NODEVICE"):  # checked before NCCL is loaded
        spj.ShardedJoin(world=1, rank=0, unique_id=bytes(128))


def test_sharded_join_argument_checks(spj):
    L = spj.lib()
    h = ctypes.c_void_p()
    uid = ctypes.create_string_buffer(128)
    d = spj.make_design()
    for world, rank in [(0, 0), (2, 2), (2, -1), (1025, 0)]:
        assert L.spj_dist_create(uid, world, rank, ctypes.byref(d), ctypes.byref(h)) == -1
    assert L.spj_dist_create(None, 1, 0, ctypes.byref(d), ctypes.byref(h)) == -1
    assert L.spj_dist_set_heavy(None, 1, 0.25, 1024) == -1
    assert L.spj_dist_heavy_keys(None, None, 0) == 0
    assert L.spj_dist_abort(None) == -1
    L.spj_dist_destroy(None)


def test_bad_arguments(spj):
    with pytest.raises(spj.SpjError, match="ARG"):
        spj.Server(1 << 30, max_batch=0)
    with pytest.raises(spj.SpjError, match="ARG"):
        spj.JoinInstance(4, 3, 1)  # ranks must equal groups x per group


def test_relation_sizes_beyond_32_bit_positions_are_rejected(spj):
    # output and partition positions are 32-bit: a relation may hold at most
    # 2^32 - 2^24 - 2 tuples; larger ones are refused before any device work
    too_big = (1 << 32) - (1 << 24) - 1
    for n_r, n_s in [(1, too_big), (too_big, 1), (1, 1 << 33)]:
        with pytest.raises(spj.SpjError, match="ARG.*2\\^32"):
            spj.Plan(n_r, n_s)
    with pytest.raises(spj.SpjError, match="ARG.*2\\^32"):
        spj.Batch([1, too_big], [1, 1])


def test_generator_relations(spj, oracle):
    R, S, expect = spj.generate_host(10000, 40000, 0.0, seed=123)
    assert sorted(R[:, 0].tolist()) == list(range(1, 10001))     # permutation of 1..n
    assert R[:, 1].tolist() == list(range(10000))                  # payload = row id
    assert S[:, 1].tolist() == list(range(40000))
    assert set(S[:, 0].tolist()) <= set(R[:, 0].tolist())          # foreign keys
    assert oracle.checksum(oracle.simple_join(R, S)) == expect


def test_generator_deterministic_across_threads(spj):
    a = spj.generate_host(3000, 7000, 1.0, seed=9, nthreads=1)
    b = spj.generate_host(3000, 7000, 1.0, seed=9, nthreads=7)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


@pytest.mark.parametrize("s", [1.0, 1.5])
def test_generator_zipf_head(spj, s):
    n, m = 1 << 14, 1 << 18
    R, S, _ = spj.generate_host(n, m, s, seed=99)
    counts = np.bincount(S[:, 0], minlength=n + 1)
    top = counts.max() / m
    h = sum(1.0 / k ** s for k in range(1, n + 1))
    assert abs(top - 1.0 / h) < 0.01, (top, 1.0 / h)


def test_cli_without_gpu_fails_loudly():
    import os
    import subprocess
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spid-join_b200", "spj_join")
    p = subprocess.run([cli, "-s", "1024", "-t", "2", "-z", "0", "-r", "1", "-R", "1", "-B", "1"],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode == 2 and "no CUDA device" in p.stderr


def test_tuning_table_roundtrip(spj):
    entries = [{"log2_r": 20, "log2_ratio": 1, "radix_bits_delta": -1, "table_slots": 8192, "unit_tuples": 0,
                "join_alg": 0},
               {"log2_r": 14, "log2_ratio": 3, "radix_bits_delta": 1, "table_slots": 0, "unit_tuples": 32768,
                "join_alg": 2}]
    spj.set_tuning(entries)
    try:
        assert spj.get_tuning() == entries
        with pytest.raises(spj.SpjError, match="ARG"):
            spj.set_tuning([{"log2_r": 20, "log2_ratio": 9}])
        assert spj.get_tuning() == entries  # a rejected table leaves the old one
    finally:
        spj.set_tuning([])
    assert spj.get_tuning() == []


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 130])
def test_dpu_block_layout(spj, n):
    """The reference's transfer layout of one rank's pairs: 64 blocks of
    ceil(n / 64) pairs, the pairs dealt evenly in order (block sizes differ by
    at most one), each block padded with (0, 0)."""
    pairs = (np.arange(2 * n, dtype=np.uint32).reshape(n, 2) + 1)
    out = spj._dpu_blocks(pairs)
    per = -(-n // 64)
    assert out.shape == (64 * per, 2)
    blocks = out.reshape(64, per, 2) if per else out.reshape(64, 0, 2)
    filled = (blocks[:, :, 0] != 0).sum(1)
    assert filled.sum() == n and (filled.max() - filled.min() <= 1 if n else True)
    assert np.array_equal(np.concatenate([blocks[b, :filled[b]] for b in range(64)]), pairs)  # order kept
    for b in range(64):
        assert not blocks[b, filled[b]:].any()  # padding is (0, 0)


C_CALLER = r"""
#include <stdio.h>
#include "spidjoin.h"

int main(void) {
    spj_design_t d;
    spj_design_default(&d);
    d.rank_num = 4;
    d.rank_set = 4;
    spj_plan_shape_t sh;
    int rc = spj_plan_describe((int64_t)1 << 27, (int64_t)1 << 29, &d, 148, 232448, 0, &sh);
    printf("describe %d %d %d %d %d\n", rc, sh.join_alg, sh.radix_bits, sh.scatter_passes, sh.table_slots);
    spj_plan_t *plan = NULL;
    rc = spj_plan_create(1000, 2000, &d, &plan);
    printf("create %d %s\n", rc, spj_last_error());
    return 0;
}
"""


def _build_dir(name):
    """A scratch directory for a test's build products inside the repository's
    git-ignored _build/."""
    d = os.path.join(ROOT, "_build", "tests", name)
    os.makedirs(d, exist_ok=True)
    return d


def test_header_compiles_as_c_and_links():
    """The boundary is a C ABI: a strict C11 program (-pedantic -Werror)
    includes include/spidjoin.h, links libspidjoin.so and calls it. The
    planner's description works without a device; a join entry point returns
    SPJ_E_NODEVICE (with no GPU) instead of running anywhere else."""
    import shutil
    import subprocess
    import torch
    cc = shutil.which("gcc") or shutil.which("cc")
    lib_dir = os.path.join(ROOT, "spid-join_b200")
    if not cc or not os.path.exists(os.path.join(lib_dir, "libspidjoin.so")):
        pytest.skip("no C compiler or library")
    d = _build_dir("c_caller")
    src, exe = os.path.join(d, "caller.c"), os.path.join(d, "caller")
    with open(src, "w") as f:
        f.write(C_CALLER)
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", lib_dir, "-lspidjoin", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60, check=True).stdout.split("\n")
    assert out[0] == "describe 0 0 15 2 12288"
    if not torch.cuda.is_available():
        assert out[1].startswith("create -7 no CUDA device")


def test_reference_driver_compiles_unchanged_against_the_facade():
    """The drop-in claim for C++ callers: the reference's own driver
    (test/join/main.cc of the reference, unmodified) compiles against
    include/pidjoin.hpp and links libspidjoin.so. Run without a GPU it stops
    with pidjoin::Error instead of computing anywhere else. Skipped where the
    reference tree is absent."""
    import shutil
    import subprocess
    import torch
    ref = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-dir"], capture_output=True,
                         text=True).stdout.strip()
    main_cc = os.path.join(ref, "test", "join", "main.cc")
    cxx = shutil.which("g++")
    lib_dir = os.path.join(ROOT, "spid-join_b200")
    if not (ref and os.path.exists(main_cc) and cxx and os.path.exists(os.path.join(lib_dir, "libspidjoin.so"))):
        pytest.skip("no reference driver, C++ compiler or library here")
    exe = os.path.join(_build_dir("reference_driver"), "ref_main")
    subprocess.run([cxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), main_cc, "-L", lib_dir, "-lspidjoin",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    if not torch.cuda.is_available():
        p = subprocess.run([str(exe), "-s", "1024", "-t", "2", "-z", "0", "-r", "1", "-R", "1", "-B", "1"],
                           capture_output=True, text=True, timeout=60)
        assert p.returncode != 0 and "no CUDA device" in p.stderr
