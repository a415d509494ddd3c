#!/usr/bin/env python
"""Runs the batch planner's autotuner on this GPU over the size classes of the
batched workload (|R| from 2^12 to 2^23, |S|/|R| from 1 to 8) and writes the
per-class table that spidjoin.load_tuning() installs:

    python spid-join_b200/autotune.py [--out spid-join_b200/tuning_b200.json] [--zipf 1.0]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import spidjoin  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tuning_b200.json"))
    ap.add_argument("--zipf", type=float, default=0.75, help="Zipf exponent of the tuning inputs")
    ap.add_argument("--log2-r", default="12-23")
    ap.add_argument("--log2-ratio", default="0-3")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    lo, hi = (int(x) for x in a.log2_r.split("-"))
    rlo, rhi = (int(x) for x in a.log2_ratio.split("-"))
    classes = [(lr, lt) for lr in range(lo, hi + 1) for lt in range(rlo, rhi + 1)]
    t0 = time.time()
    table = spidjoin.autotune(classes, zipf=a.zipf, reps=a.reps, log=lambda e: print(json.dumps(e), flush=True))
    import torch
    out = {"device": torch.cuda.get_device_name(0), "zipf": a.zipf, "reps": a.reps,
           "seconds": round(time.time() - t0, 1), "entries": table}
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {a.out}: {len(table)} classes in {out['seconds']} s")


if __name__ == "__main__":
    main()
