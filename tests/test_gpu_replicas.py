"""Replica sets: many independent trees of uneven size run their Metropolis
sequences in one launch (one block per tree). Each replica must reproduce its
own single-tree run: the same accept decisions and final positions, energy
shifts within the parity tolerance, and maintained energies that match; two
replicas are also replayed move by move on the oracle's tree."""
import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ABS_DE = 2e-10
REL_E = 1e-11


def system(n, seed):
    rng = np.random.default_rng(seed)
    L = n ** (1 / 3)
    return rng.uniform(0, L, 3 * n), np.where(np.arange(n) % 2 == 0, 1.0, -1.0), L


@pytest.mark.parametrize("digits", [6, 9])
def test_replicas_match_single_tree_runs(digits):
    sizes = [2000, 3500, 6000, 9000, 15000, 24000]
    m = 64
    rng = np.random.default_rng(100 + digits)
    reps, twins, moves, oracles = [], [], [], []
    for k, n in enumerate(sizes):
        r, q, L = system(n, k)
        npl = max(16, n // 128)  # depth >= 3 for every replica
        prm = P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT)
        a = P.HPDMKPtTree(prm, r, q, leaf_slack=4)
        b = P.HPDMKPtTree(prm, r, q, leaf_slack=4)
        for t in (a, b):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        reps.append(a)
        twins.append(b)
        if k < 2:
            o = O.OracleTree(L, npl, digits, r, q)
            o.form_outgoing_pw()
            o.form_incoming_pw()
            oracles.append(o)
        moves.append((rng.integers(0, n, m), rng.uniform(-0.3, 0.3, (m, 3)), rng.uniform(0, 1, m)))
    try:
        idx = np.stack([mv[0] for mv in moves])
        disp = np.stack([mv[1] for mv in moves])
        u = np.stack([mv[2] for mv in moves])
        dE, acc = P.replicas_mc_run(reps, idx, disp, u, 1.0)
        for k, o in enumerate(oracles):
            for c in range(m):
                de = o.eval_shift_energy(int(idx[k, c]), *disp[k, c])
                assert abs(dE[k, c] - de) <= ABS_DE * max(1.0, abs(de)), (k, c, dE[k, c], de)
                assert bool(acc[k, c]) == bool(u[k, c] < np.exp(-de)), (k, c)
                if acc[k, c]:
                    o.update_shift(int(idx[k, c]), *disp[k, c])
            np.testing.assert_array_equal(reps[k].positions(), o.positions())
        for k in range(len(sizes)):
            d1, a1 = twins[k].mc_run(moves[k][0], moves[k][1], moves[k][2], 1.0)
            np.testing.assert_array_less(np.abs(dE[k] - d1), ABS_DE * np.maximum(1.0, np.abs(d1)))
            np.testing.assert_array_equal(acc[k], a1)
            np.testing.assert_array_equal(reps[k].positions(), twins[k].positions())
            e1, e2 = reps[k].eval_energy(), twins[k].eval_energy()
            assert abs(e1 - e2) <= REL_E * abs(e2)
        assert 0 < acc.mean() < 1
        # replica energies, several trees in flight, equal the trees' own
        np.testing.assert_array_equal(P.replicas_energy(reps), [t.eval_energy() for t in reps])
        # a second batch continues from the updated states
        dE2, acc2 = P.replicas_mc_run(reps, idx[:, ::-1], disp, u, 1.0)
        for k in range(len(sizes)):
            d1, a1 = twins[k].mc_run(idx[k, ::-1], disp[k], u[k], 1.0)
            np.testing.assert_array_equal(acc2[k], a1)
            np.testing.assert_array_less(np.abs(dE2[k] - d1), ABS_DE * np.maximum(1.0, np.abs(d1)))
    finally:
        for t in reps + twins:
            t.close()


def test_replicas_reject_mixed_digits():
    r, q, L = system(2000, 1)
    a = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=20, digits=6, L=L, init=P.DIRECT), r, q)
    b = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=20, digits=9, L=L, init=P.DIRECT), r, q)
    try:
        for t in (a, b):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        with pytest.raises(P.HPDMKError):
            P.replicas_mc_run([a, b], np.zeros((2, 4), np.int64), np.zeros((2, 4, 3)), np.zeros((2, 4)), 1.0)
    finally:
        a.close()
        b.close()
