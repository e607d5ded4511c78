"""Ewald energy of the bench workload, computed once on the CPU by the
oracle's FP64 Ewald (s = 5, alpha = 0.4; about 90 s on 8 cores) and stored in
tests/golden/bench_ewald.json. bench.py reports the DMK energy's relative
error against it, and a GPU test checks the library's own Ewald against it.

    make -C oracle && python tests/golden/make_bench_ewald.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    W = bench.WORKLOAD_N1E5
    r, q = bench.make_system(1, W["N"], W["L"])
    e = O.ewald_energy(W["L"], r, q, s=5.0, alpha=0.4)
    out = {"workload": {"N": W["N"], "L": W["L"], "seed": 1, "charges": "alternating +1/-1"},
           "ewald": {"s": 5.0, "alpha": 0.4, "energy": e},
           "note": "E = 1/2 sum' q_i q_j / r over periodic images (no 4 pi), as the DMK energy"}
    with open(os.path.join(HERE, "bench_ewald.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(e)


if __name__ == "__main__":
    main()
