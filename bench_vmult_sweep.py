"""Operator-application sweep over FE degrees 1..6 on the unit cube, affine and
deformed (interior vertices perturbed by up to 0.2 h), FP64 and FP32, constant
coefficients: the vmult throughput table.

  python bench_vmult_sweep.py [--size large|small] [--reps 10]

Meshes hold ~64 M (large) or ~2 M (small) DoFs: 399/125 cells per direction at
p = 1, 199/62 (p = 2), 133/42 (3), 100/31 (4), 80/25 (5), 66/21 (6). Each case runs
in its own process (bench_vmult.py); prints one JSON line per case and a markdown
table with GDoF/s, algorithmic GB/s (src + dst [+ 7 per-q geometry factors]) and
its fraction of the measured HBM bandwidth.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

CELLS = {"large": {1: 399, 2: 199, 3: 133, 4: 100, 5: 80, 6: 66},
         "small": {1: 125, 2: 62, 3: 42, 4: 31, 5: 25, 6: 21}}


def hbm_peak():
    try:
        return float(json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default="large", choices=list(CELLS))
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args()
    peak = hbm_peak()
    rows = []
    for p, m in CELLS[a.size].items():
        for perturb in (0.0, 0.2):
            r = subprocess.run([sys.executable, os.path.join(HERE, "bench_vmult.py"), "--degree",
                                str(p), "--cells", str(m), "--perturb", str(perturb), "--law", "0",
                                "--reps", str(a.reps), "--dtype", "both"],
                               capture_output=True, text=True)
            if r.returncode != 0:
                print(r.stdout + r.stderr, file=sys.stderr)
                return r.returncode
            for line in r.stdout.splitlines():
                if line.startswith("{"):
                    d = json.loads(line)
                    print(line, flush=True)
                    rows.append(d)
    print("\n| p | cells | geometry | dtype | ms | GDoF/s | alg GB/s | of HBM |")
    print("|---|---|---|---|---|---|---|---|")
    for d in rows:
        print(f"| {d['degree']} | {d['cells']}^3 | {'deformed' if d['perturb'] else 'affine'} | "
              f"{d['dtype']} | {d['ms']:.3f} | {d['gdofs']:.1f} | {d['alg_gbs']:.0f} | "
              f"{d['alg_gbs'] / peak:.0%} |")
    return 0


if __name__ == "__main__":
    sys.exit(main())
