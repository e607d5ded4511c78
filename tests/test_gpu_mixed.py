"""Mixed precision (HPDMK_PRECISION_MIXED): the outgoing plane-wave
expansions formed on the tensor cores (tcgen05 kind::i8) from four signed
8-bit slices (a 32-bit fixed point) of each phase-factor product, against the oracle's FP64 expansions (the
reference's nudft3d1_halfplane, include/nudft.hpp:95-121, and the root pass,
src/planewave.cpp:24-46); the energies and energy shifts that follow from
them against the oracle and the FP64 Ewald energy."""
import json
import os

import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

# Each slice product is exact (32-bit integer sums); an operand carries the
# rounding of its 32-bit fixed point (2.3e-10 of its range for B, at most
# twice that for A, whose components round twice: |factor| <= 1, charges
# scaled by max |q|) and the ten-product truncation (zero-mean, below
# 1e-9 of the range), so a coefficient of a box of n random-phase particles
# is off by about sqrt(n) 4e-10: the bound below is relative to the largest
# coefficient of the box.
REL_PW_MIXED = 2e-8
ABS_DE_MIXED = 1e-8


def rel_e_mixed(digits):
    """Mixed energy against the FP64 energy, relative to |E|: the 1e-8 target
    at 9 and 12 digits; at 3 and 6 digits a tenth of the method's own error."""
    return 1e-8 if digits >= 9 else 10.0 ** -(digits + 1)


def system(kind, n, L, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        r = rng.uniform(0, L, (n, 3))
    elif kind == "clustered":
        c = rng.uniform(0, L, (6, 3))
        m = int(0.8 * n)
        r = np.concatenate([np.mod(c[rng.integers(0, 6, m)] + rng.normal(0, L / 40, (m, 3)), L),
                            rng.uniform(0, L, (n - m, 3))])
    elif kind == "reference":
        return O.reference_test_system(n, L)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return np.ascontiguousarray(r.reshape(-1)), q


CASES = [
    # (kind, n, L, n_per_leaf, digits): every supported digits setting, so
    # every mode count of the mixed kernel (window and difference) runs
    ("uniform", 1000, 10.0, 10, 6),      # the reference's first configuration
    ("reference", 1000, 20.0, 10, 3),
    ("clustered", 6000, 20.0, 20, 9),
    ("uniform", 3000, 46.4, 8, 12),
]


def mixed_tree(r, q, L, npl, digits, slack=8):
    return P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT), r, q,
                         leaf_slack=slack, precision=P.PRECISION_MIXED)


@pytest.mark.parametrize("case", CASES)
def test_mixed_expansions_and_energy(case):
    kind, n, L, npl, digits = case
    r, q = system(kind, n, L)
    g = mixed_tree(r, q, L, npl, digits)
    o = O.OracleTree(L, npl, digits, r, q)
    try:
        for t in (g, o):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        ro, rg = o.pw(0), g.pw(0)
        assert np.abs(rg - ro).max() <= REL_PW_MIXED * np.abs(ro).max(), np.abs(rg - ro).max() / np.abs(ro).max()
        lv, pf, leaf, cnt = o.tree_nodes()
        worst = 0.0
        for node in np.nonzero((lv >= 2) & (lv <= o.max_depth - 2))[0][:300]:
            a, b = g.pw(node), o.pw(node)
            scale = max(np.abs(b).max(), 1e-300)
            worst = max(worst, np.abs(a - b).max() / scale)
        assert worst <= REL_PW_MIXED, worst
        pg, po = g.eval_energy_parts(), o.eval_energy_parts()
        E = po.sum()
        rel = abs(pg.sum() - E) / abs(E)
        print(f"\nACCURACY mixed {case}: pw {worst:.2e} (root {np.abs(rg - ro).max() / np.abs(ro).max():.2e}), "
              f"energy vs FP64 oracle {rel:.3e}, parts {pg - po}")
        assert rel <= rel_e_mixed(digits), (pg, po, rel)
        # the near field does not depend on the expansions: unchanged
        assert abs(pg[2] - po[2]) <= 1e-11 * abs(E)
    finally:
        g.close()


def test_mixed_shifts_updates_and_metropolis():
    # energy shifts read the incoming expansions that the mixed pass formed;
    # the shift itself and the update stay FP64
    r, q = system("clustered", 6000, 20.0, seed=2)
    g = mixed_tree(r, q, 20.0, 20, 9)
    o = O.OracleTree(20.0, 20, 9, r, q)
    try:
        for t in (g, o):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        rng = np.random.default_rng(3)
        for step in range(16):
            i = int(rng.integers(0, 6000))
            d = rng.uniform(-0.5, 0.5, 3)
            dg = g.eval_shift_energy(i, *d)
            do = o.eval_shift_energy(i, *d)
            assert abs(dg - do) <= ABS_DE_MIXED * max(1.0, abs(do)), (step, dg, do)
            if step % 2 == 0:
                g.update_shift(i, *d)
                o.update_shift(i, *d)
        m = 200
        idx = rng.integers(0, 6000, m)
        disp = rng.uniform(-0.3, 0.3, (m, 3))
        u = rng.uniform(0, 1, m)
        dEm, acc = g.mc_run(idx, disp, u, 1.0)
        for c in range(m):
            de = o.eval_shift_energy(int(idx[c]), *disp[c])
            assert abs(dEm[c] - de) <= ABS_DE_MIXED * max(1.0, abs(de)), (c, dEm[c], de)
            # the same decision (no move sits within 1e-8 of the threshold here)
            assert bool(acc[c]) == bool(u[c] < np.exp(-de)), c
            if acc[c]:
                o.update_shift(int(idx[c]), *disp[c])
        np.testing.assert_array_equal(g.positions(), o.positions())
        # a new outgoing pass on the moved particles
        g.form_outgoing_pw()
        g.form_incoming_pw()
        o.form_outgoing_pw()
        o.form_incoming_pw()
        E, Eo = g.eval_energy(), o.eval_energy()
        assert abs(E - Eo) <= rel_e_mixed(9) * abs(Eo), (E, Eo)
    finally:
        g.close()


def test_mixed_bench_workload_vs_ewald():
    # uniform N = 1e5, L = 46.4, 9 digits: the mixed energy against the stored
    # FP64 Ewald energy of the same positions, at the 1e-8 target
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    import bench
    gl = json.load(open(os.path.join(HERE, "golden", "bench_ewald.json")))
    W = bench.WORKLOAD_N1E5
    r, q = bench.make_system(1, W["N"], W["L"])
    assert gl["workload"]["N"] == W["N"] and gl["workload"]["L"] == W["L"] and gl["workload"]["seed"] == 1
    params = P.HPDMKParams(n_per_leaf=W["n_per_leaf"], digits=W["digits"], L=W["L"], init=P.DIRECT)
    g = P.HPDMKPtTree(params, r, q, precision=P.PRECISION_MIXED)
    f = P.HPDMKPtTree(params, r, q)
    try:
        for t in (g, f):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        Em, Ef = g.eval_energy(), f.eval_energy()
        ew = gl["ewald"]["energy"]
        print(f"\nACCURACY N=1e5 cube: mixed vs Ewald {abs(Em - ew) / abs(ew):.3e}, FP64 vs Ewald "
              f"{abs(Ef - ew) / abs(ew):.3e}, mixed vs FP64 {abs(Em - Ef) / abs(Ef):.3e}")
        assert abs(Em - ew) <= 1e-8 * abs(ew), (Em, ew, abs(Em - ew) / abs(ew))
        assert abs(Em - Ef) <= 1e-8 * abs(Ef), (Em, Ef)
    finally:
        g.close()
        f.close()


def test_mixed_largest_split_k_chunk():
    # one level-2 box holds 20 000 particles, so with ksplit = 16384 one
    # split-K chunk carries the most particles the exact int32 sums allow;
    # expansions and energy against the FP64 path (parity-tested against the
    # oracle elsewhere)
    rng = np.random.default_rng(9)
    L, n_in, n_out = 24.0, 20000, 4000
    r = np.concatenate([rng.uniform(0.5, 5.5, (n_in, 3)), rng.uniform(0, L, (n_out, 3))])
    r = np.ascontiguousarray(r.reshape(-1))
    n = n_in + n_out
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    prm = P.HPDMKParams(n_per_leaf=400, digits=9, L=L, init=P.DIRECT)
    g = P.HPDMKPtTree(prm, r, q, precision=P.PRECISION_MIXED)
    f = P.HPDMKPtTree(prm, r, q)
    try:
        g.set_tuning(ksplit=16384, ksplit_root=16384)
        assert g.tuning()["ksplit"] == 16384
        for t in (g, f):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        rg, rf = g.pw(0), f.pw(0)
        assert np.abs(rg - rf).max() <= REL_PW_MIXED * np.abs(rf).max()
        lv, pf, leaf, cnt = O.OracleTree(L, 400, 9, r, q).tree_nodes()
        big = [int(b) for b in np.nonzero((lv == 2) & (cnt > 16384))[0]]
        assert big, "no box above the chunk size"
        for b in big:
            a, c = g.pw(b), f.pw(b)
            assert np.abs(a - c).max() <= REL_PW_MIXED * np.abs(c).max()
        Em, Ef = g.eval_energy(), f.eval_energy()
        assert abs(Em - Ef) <= rel_e_mixed(9) * abs(Ef), (Em, Ef)
    finally:
        g.close()
        f.close()


def test_mixed_edge_cases():
    """The mixed path at the edges the FP64 parity test covers: a single
    charge (its periodic self-image energy, against the oracle), boundary
    coordinates and a multi-box wrap (against the FP64 tree and the oracle),
    and a system of zero charges, whose fixed-point scale max|q| is zero (every
    expansion, energy and shift exactly zero)."""
    L = 8.0
    r1, q1 = np.array([1.0, 2.0, 3.0]), np.array([1.0])
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=4, digits=9, L=L, init=P.DIRECT), r1, q1,
                      precision=P.PRECISION_MIXED)
    o = O.OracleTree(L, 4, 9, r1, q1)
    try:
        for t in (g, o):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        Eg, Eo = g.eval_energy(), o.eval_energy()
        assert abs(Eg - Eo) <= rel_e_mixed(9) * max(1.0, abs(Eo)), (Eg, Eo)
        assert abs(g.eval_shift_energy(0, 1.5, -2.0, 7.9)) <= ABS_DE_MIXED
    finally:
        g.close()

    rng = np.random.default_rng(4)
    r = rng.uniform(0, L, (500, 3))
    r[0] = [0.0, 0.0, 0.0]
    r[1] = [np.nextafter(L, 0), np.nextafter(L, 0), 0.0]
    r[2] = [L / 2, L / 4, L / 8]
    r = np.ascontiguousarray(r.reshape(-1))
    q = np.where(np.arange(500) % 2 == 0, 1.0, -1.0)
    params = P.HPDMKParams(n_per_leaf=6, digits=9, L=L, init=P.DIRECT)
    g = P.HPDMKPtTree(params, r, q, precision=P.PRECISION_MIXED)
    f = P.HPDMKPtTree(params, r, q, precision=P.PRECISION_FP64)
    o = O.OracleTree(L, 6, 9, r, q)
    try:
        for t in (g, f, o):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        Eo = o.eval_energy()
        assert abs(g.eval_energy() - Eo) <= rel_e_mixed(9) * abs(Eo), (g.eval_energy(), Eo)
        for i, d in [(0, (L, 0.0, 0.0)), (1, (1e-9, 0.0, -1e-9)), (2, (0.0, 0.0, 0.0)),
                     (3, (-2.5 * L, 3.25 * L, 0.5))]:
            dg, df, do = g.eval_shift_energy(i, *d), f.eval_shift_energy(i, *d), o.eval_shift_energy(i, *d)
            assert abs(dg - df) <= ABS_DE_MIXED * max(1.0, abs(df)), (i, d, dg, df)
            assert abs(dg - do) <= ABS_DE_MIXED * max(1.0, abs(do)), (i, d, dg, do)
            for t in (g, f, o):
                t.update_shift(i, *d)
        np.testing.assert_array_equal(g.positions(), o.positions())
        Eg, Ef = g.eval_energy(), f.eval_energy()
        assert abs(Eg - Ef) <= rel_e_mixed(9) * abs(Ef), (Eg, Ef)
    finally:
        g.close()
        f.close()

    q0 = np.zeros(500)
    g = P.HPDMKPtTree(params, r, q0, precision=P.PRECISION_MIXED)
    try:
        g.form_outgoing_pw()
        g.form_incoming_pw()
        assert g.eval_energy() == 0.0
        assert g.eval_shift_energy(7, 0.3, -0.2, 0.1) == 0.0
    finally:
        g.close()
