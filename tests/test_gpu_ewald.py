"""The library's FP64 GPU Ewald comparator against the oracle's CPU Ewald
(small systems and the bench workload's stored value), and the DMK energy
against it at the reference's tolerance 5e-(d-1) |E| (test/hpdmk_test.cpp,
compare_energy), up to N = 1e6 where a CPU Ewald is impractical."""
import json
import os

import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REL_EWALD = 1e-10  # GPU against CPU Ewald, both truncated near 1e-12


def tree(r, q, L, digits=9, npl=20):
    return P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT), r, q, leaf_slack=4)


@pytest.mark.parametrize("n,L,seed", [(2000, 12.6, 1), (5000, 17.1, 2), (3000, 14.4, 3)])
def test_gpu_ewald_vs_oracle(n, L, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = tree(r, q, L)
    try:
        e, parts = t.ewald_energy()
        assert abs(parts.sum() - e) <= 1e-12 * abs(e)
        ref = O.ewald_energy(L, r, q, s=5.0, alpha=1.0)
        assert abs(e - ref) <= REL_EWALD * abs(ref), (e, ref)
        # after moves the comparator follows the particles
        idx = rng.choice(n, 50, replace=False)
        disp = rng.uniform(-0.5, 0.5, (50, 3))
        for i, d in zip(idx, disp):
            t.eval_shift_energy(int(i), *d)
            t.update_shift(int(i), *d)
        e2, _ = t.ewald_energy()
        ref2 = O.ewald_energy(L, np.ascontiguousarray(t.positions()), q, s=5.0, alpha=1.0)
        assert abs(e2 - ref2) <= REL_EWALD * abs(ref2)
    finally:
        t.close()


def test_gpu_ewald_bench_workload_and_dmk_error():
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    import bench
    g = json.load(open(os.path.join(HERE, "golden", "bench_ewald.json")))
    W = bench.WORKLOAD_N1E5
    r, q = bench.make_system(1, W["N"], W["L"])
    t = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=W["n_per_leaf"], digits=W["digits"], L=W["L"], init=P.DIRECT), r, q)
    try:
        e, _ = t.ewald_energy()
        assert abs(e - g["ewald"]["energy"]) <= REL_EWALD * abs(e)
        t.form_outgoing_pw()
        t.form_incoming_pw()
        dmk = t.eval_energy()
        assert abs(dmk - e) <= 5 * 10.0 ** (-W["digits"] + 1) * abs(e)
    finally:
        t.close()


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_dmk_vs_gpu_ewald_digits(digits):
    n, L = 20000, 27.1
    rng = np.random.default_rng(digits)
    r = rng.uniform(0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = tree(r, q, L, digits=digits, npl=50)
    try:
        e, _ = t.ewald_energy()
        t.form_outgoing_pw()
        t.form_incoming_pw()
        dmk = t.eval_energy()
        assert abs(dmk - e) <= 5 * 10.0 ** (-digits + 1) * abs(e), (digits, dmk, e)
    finally:
        t.close()


def clustered(n, L, seed, n_clusters=64, frac=0.8):
    """64 isotropic Gaussian clusters (centres uniform, sigma = L/40) plus a 20 % uniform background."""
    rng = np.random.default_rng(seed)
    m = int(frac * n)
    c = rng.uniform(0, L, (n_clusters, 3))
    r = np.concatenate([np.mod(c[rng.integers(0, n_clusters, m)] + rng.normal(0, L / 40, (m, 3)), L),
                        rng.uniform(0, L, (n - m, 3))])
    r[r >= L] = 0.0  # a wrap that rounds to L
    return np.ascontiguousarray(r.reshape(-1))


# The target accuracy at N = 1e6: 1e-8 relative to the FP64 Ewald energy, for
# the FP64 path and the mixed-precision path, on the uniform cube (the
# candidate-query configuration, 9 digits) and the clustered system. On the
# clustered system 9 digits give the method's own error near 2e-8 (inside
# the reference's 5e-8 tolerance at 9 digits, checked here), so the 1e-8
# target takes 12 digits there, the escalation the workload allows.
@pytest.mark.parametrize("kind,digits,tol", [("uniform", 9, 1e-8), ("clustered", 9, 5e-8), ("clustered", 12, 1e-8)])
@pytest.mark.parametrize("precision", [P.PRECISION_FP64, P.PRECISION_MIXED])
def test_dmk_vs_gpu_ewald_n1e6(kind, digits, tol, precision):
    n, L = 1_000_000, 100.0
    rng = np.random.default_rng(21)
    r = rng.uniform(0, L, 3 * n) if kind == "uniform" else clustered(n, L, 21)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=200, digits=digits, L=L, init=P.DIRECT), r, q, leaf_slack=0,
                      precision=precision)
    try:
        e, _ = t.ewald_energy()
        t.form_outgoing_pw()
        t.form_incoming_pw()
        dmk = t.eval_energy()
        rel = abs(dmk - e) / abs(e)
        print(f"\nACCURACY n1e6 {kind} digits={digits} precision={precision} depth={t.max_depth} dmk={dmk!r} "
              f"ewald={e!r} rel={rel:.3e}")
        assert rel <= tol, (dmk, e, rel)
    finally:
        t.close()
