"""Writes kat_main_cc.json: known answers for the reference's own synthetic test,
test/join/main.cc:30-43 of yonsei-hpcp/spid-join (R.key = i+1, R.pay = i+3;
S.key = i/ratio + 1, S.pay = i/ratio + 3). Every S tuple matches exactly one R
tuple, so the join is {(k+2, k+2) x ratio : k = 1..N}. The answers are derived
from that formula here, independently of the oracle and of the GPU code."""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def case(n, ratio):
    s = 0
    for k in range(1, n + 1):
        v = ((k + 2) << 32) | (k + 2)
        s = (s + ratio * mix64(v)) & M64
    return {"N": n, "ratio": ratio, "n_pairs": n * ratio, "checksum": s,
            "first_sorted": [[3, 3]] * min(ratio, 4)}


def main():
    cases = [case(n, r) for n, r in [(1, 1), (100, 1), (1000, 2), (4096, 8), (65536, 2), (100003, 3)]]
    with open(os.path.join(HERE, "kat_main_cc.json"), "w") as f:
        json.dump({"source": "test/join/main.cc:30-43", "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
