"""The command-line driver spj_join, run with the reference driver's knobs
(test/join/main.cc:73-118: -s -r -z -t -R -B): it joins through the pidjoin.hpp
facade and checks its output's count and checksum itself (exit status 0)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spid-join_b200", "spj_join")


@pytest.mark.parametrize("args", [
    "-s 1048576 -t 2 -z 0 -r 1 -R 1 -B 1",          # the reference's small configuration
    "-s 262144 -t 4 -z 100 -r 4 -R 4 -B 1",          # Zipf 1.0, replication groups of 4
    "-s 65536 -t 8 -z 150 -r 4 -R 1 -B 16 -a smj",
    "-s 65536 -t 2 -z 50 -r 2 -R 2 -B 1 -a nl",
    "-s 100000 -t 3 -z 0 -r 1 -R 1 -B 1 -a nphj -n 2",
    "-s 200000 -t 2 -z 120 -r 4 -R 2 -B 1 -n 2 -o",  # result buffers owned (and freed) by the caller
    "-s 100003 -t 3 -z 0 -r 4 -R 2 -B 1 -P",         # the reference's padded 64-block layout
])
def test_cli_joins_and_verifies(args):
    p = subprocess.run([CLI] + args.split(), capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "check: ok" in p.stdout and "MISMATCH" not in p.stdout


def test_cli_padded_layout_sizes():
    """-P: every rank's buffer is 64 blocks of one size, so its byte size is a
    multiple of 64 * 8, and the padding adds less than 64 pairs per rank."""
    import re
    n_s = 100003 * 3
    p = subprocess.run([CLI] + "-s 100003 -t 3 -z 0 -r 4 -R 2 -B 1 -P".split(), capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    m = re.search(r"padded layout: (\d+) bytes in (\d+) ranks", p.stdout)
    assert m, p.stdout
    total, ranks = int(m.group(1)), int(m.group(2))
    assert ranks == 4 and total % 512 == 0 and 8 * n_s <= total < 8 * n_s + ranks * 64 * 8


def test_sharded_join_from_cpp():
    """spj_dist_check: the sharded join's C sequence (NCCL id, create, heavy keys,
    join twice, destroy) from a C++ program with no Python, on one rank; the
    pairs match the generator's count and checksum."""
    exe = os.path.join(os.path.dirname(CLI), "spj_dist_check")
    p = subprocess.run([exe, str(1 << 18), str(1 << 21), "1.5"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.count("check: ok") == 2 and "heavy_keys=0" not in p.stdout
