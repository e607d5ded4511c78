"""Fill the autotuner's table for the uniform periodic cubes at density 1:
for each (N, precision) a tree is built from seeded uniform positions with
alternating +1/-1 charges and hpdmk_autotune searches its run-time splits
and tiles (see include/hpdmk.h).

    python -m pdmk4mc_b200.autotune [--out tuning.json] [--digits 9] [--n 100000 1000000]
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from .tree import DIRECT, PRECISION_FP64, PRECISION_MIXED, HPDMKParams, HPDMKPtTree


def tune_cube(n, digits, precision, out, n_per_leaf=200, reps=3):
    L = n ** (1.0 / 3.0)
    rng = np.random.default_rng(1)
    r = rng.uniform(0.0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = HPDMKPtTree(HPDMKParams(n_per_leaf=n_per_leaf, digits=digits, L=L, init=DIRECT), r, q, leaf_slack=0,
                    precision=precision)
    try:
        return t.autotune(out, reps=reps)
    finally:
        t.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None, help="table file (default: tuning.json beside the library)")
    ap.add_argument("--digits", type=int, default=9)
    ap.add_argument("--n", type=int, nargs="+", default=[100000, 1000000])
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    for n in a.n:
        for prec in (PRECISION_FP64, PRECISION_MIXED):
            chosen, times = tune_cube(n, a.digits, prec, a.out, reps=a.reps)
            print(json.dumps({"N": n, "digits": a.digits, "precision": prec, "chosen": chosen, "ms": times}))


if __name__ == "__main__":
    main()
