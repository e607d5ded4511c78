"""Tree maintenance: after many accepted moves (leaves drift from n_per_leaf
and arrivals overflow into the pool), hpdmk_tree_rebuild re-bins the tree on
the device. The rebuilt tree must equal a tree built from the current
positions: the same nodes, neighbour lists and particle order, the same
energies and energy shifts, and the same Metropolis run afterwards; and it
must match the oracle's tree built from those positions (nodes, neighbour
lists and order bit for bit, energy parts to the parity tolerance)."""
import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

REL_E = 1e-11

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [P.MC_PERSISTENT, P.MC_GRAPH])
def test_rebuild_equals_fresh_tree(mode):
    n, L, npl, digits = 4000, 16.0, 10, 9
    rng = np.random.default_rng(12)
    c = rng.uniform(0, L, (4, 3))
    r = np.mod(c[rng.integers(0, 4, n)] + rng.normal(0, L / 10, (n, 3)), L)
    r[r >= L] = 0.0
    r = np.ascontiguousarray(r.reshape(-1))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    params = P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT)
    t = P.HPDMKPtTree(params, r, q, leaf_slack=1, pool_capacity=4096)
    t.set_mc_mode(mode)
    t.form_outgoing_pw()
    t.form_incoming_pw()
    m = 800
    idx = rng.integers(0, n, m)
    disp = rng.uniform(-1.5, 1.5, (m, 3))
    u = rng.uniform(0, 1, m)
    _, acc = t.mc_run(idx, disp, u, 0.05)  # hot: most moves accepted
    assert acc.mean() > 0.5
    t.rebuild()
    pos = np.ascontiguousarray(t.positions())
    f = P.HPDMKPtTree(params, pos, q, leaf_slack=1, pool_capacity=4096)
    f.set_mc_mode(mode)
    f.form_outgoing_pw()
    f.form_incoming_pw()
    o = O.OracleTree(L, npl, digits, pos, q)
    o.form_outgoing_pw()
    o.form_incoming_pw()
    try:
        assert (t.max_depth, t.n_nodes) == (o.max_depth, o.n_nodes)
        for a, b in zip(t.tree_nodes(), o.tree_nodes()):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(t.tree_neighbors(), o.tree_neighbors()):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(t.sorted_order(), o.sorted_order())
        pt, po = t.eval_energy_parts(), o.eval_energy_parts()
        assert np.all(np.abs(pt - po) <= REL_E * abs(po.sum())), (pt, po)
        assert (t.max_depth, t.n_nodes) == (f.max_depth, f.n_nodes)
        for a, b in zip(t.tree_nodes(), f.tree_nodes()):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(t.tree_neighbors(), f.tree_neighbors()):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(t.sorted_order(), f.sorted_order())
        np.testing.assert_array_equal(t.eval_energy_parts(), f.eval_energy_parts())
        i2 = rng.integers(0, n, 64)
        d2 = rng.uniform(-0.5, 0.5, (64, 3))
        np.testing.assert_array_equal(t.eval_shift_energy_batch(i2, d2), f.eval_shift_energy_batch(i2, d2))
        i3 = rng.integers(0, n, 200)
        d3 = rng.uniform(-0.5, 0.5, (200, 3))
        u3 = rng.uniform(0, 1, 200)
        dt, at = t.mc_run(i3, d3, u3, 1.0)
        df, af = f.mc_run(i3, d3, u3, 1.0)
        np.testing.assert_array_equal(dt, df)
        np.testing.assert_array_equal(at, af)
        np.testing.assert_array_equal(t.positions(), f.positions())
    finally:
        t.close()
        f.close()


def test_rebuild_policy():
    # particles pulled into one corner: leaves there overfill, so with the
    # policy set the next full energy re-bins the tree first; its energy then
    # equals a fresh tree of the moved positions, and without drift nothing
    # is rebuilt
    n, L, npl, digits = 3000, 12.0, 10, 6
    rng = np.random.default_rng(41)
    r = np.ascontiguousarray(rng.uniform(0, L, 3 * n))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    params = P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT)
    t = P.HPDMKPtTree(params, r, q, leaf_slack=2, pool_capacity=8192)
    try:
        t.set_rebuild_policy(2.0)
        t.form_outgoing_pw()
        t.form_incoming_pw()
        assert t.drift()[2] == 0
        depth0 = t.max_depth
        # move 600 particles towards the corner (1, 1, 1), all accepted (beta = 0)
        idx = rng.choice(n, 600, replace=False)
        pos = t.positions().reshape(-1, 3)
        target = rng.uniform(0.5, 1.5, (600, 3))
        disp = target - pos[idx]
        _, acc = t.mc_run(idx, disp, np.zeros(600), 0.0)
        assert acc.all()
        mx, mn, nreb = t.drift()
        assert mx > 2 * npl and nreb == 0
        t.form_outgoing_pw()
        t.form_incoming_pw()
        E = t.eval_energy()
        mx2, _, nreb = t.drift()
        assert nreb == 1 and mx2 <= npl and t.max_depth > depth0
        f = P.HPDMKPtTree(params, np.ascontiguousarray(t.positions()), q)
        try:
            f.form_outgoing_pw()
            f.form_incoming_pw()
            Ef = f.eval_energy()
        finally:
            f.close()
        assert abs(E - Ef) <= REL_E * abs(Ef), (E, Ef)
        # no drift since: no second rebuild
        t.form_outgoing_pw()
        assert t.drift()[2] == 1
        with pytest.raises(P.HPDMKError):
            t.set_rebuild_policy(0.5)
    finally:
        t.close()
