"""GPU parity: the CUDA path (through the C-ABI) against the oracle on the same
seeded inputs — tree and neighbour lists bit-exact, expansions, energies,
energy shifts, sequential accept-and-update, batched and Monte Carlo calls,
overflow handling, and the reference's own Ewald scenarios."""
import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# FP64 against FP64 with different summation orders and box-centred phases:
REL_E = 1e-11     # energies, relative to |E|
ABS_DE = 2e-10    # energy shifts, absolute (shift magnitudes are O(1))
REL_PW = 1e-11    # expansions, relative to the largest coefficient


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
        r, q = O.reference_test_system(n, L)
        return r, q
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return np.ascontiguousarray(r.reshape(-1)), q


def pair(kind, n, L, npl, digits, slack=8, seed=0):
    r, q = system(kind, n, L, seed)
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT), r, q, leaf_slack=slack)
    o = O.OracleTree(L, npl, digits, r, q)
    return g, o, r, q


CASES = [
    ("uniform", 2000, 10.0, 10, 6),
    ("clustered", 6000, 20.0, 20, 9),
    ("reference", 1000, 20.0, 10, 3),
    ("uniform", 40, 5.0, 10, 6),       # shallow: every leaf at level 2, no difference levels
    ("uniform", 3000, 46.4, 8, 12),
]


def test_tree_bit_exact_deep():
    # a tight cluster refines down to the deepest allowed level: the levels
    # past the first read-back of the refinement counts, and the level cap
    rng = np.random.default_rng(4)
    L, n = 10.0, 3000
    r = np.concatenate([np.mod(np.array([3.0, 6.0, 4.5]) + rng.normal(0, L / 3000, (2000, 3)), L),
                        rng.uniform(0, L, (n - 2000, 3))]).reshape(-1)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=10, digits=6, L=L, init=P.DIRECT), r, q)
    o = O.OracleTree(L, 10, 6, r, q)
    assert g.max_depth == o.max_depth and g.max_depth >= 10
    assert g.n_nodes == o.n_nodes
    for a, b in zip(g.tree_nodes(), o.tree_nodes()):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(g.tree_neighbors(), o.tree_neighbors()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(g.sorted_order(), o.sorted_order())
    g.close()


def test_device_inputs_rejected_then_accepted():
    # positions already on the device are checked on the device during the
    # build: outside [0, L) or a non-finite charge is HPDMK_ERR_BAD_INPUT, and
    # a valid build afterwards gives the host-input tree's energy
    import torch
    L, n = 10.0, 2000
    r, q = system("uniform", n, L, seed=3)
    params = P.HPDMKParams(n_per_leaf=10, digits=6, L=L, init=P.DIRECT)
    bad_r = r.copy()
    bad_r[3 * 17 + 1] = L  # one coordinate at L, outside [0, L)
    bad_q = q.copy()
    bad_q[5] = np.nan
    for rr, qq in ((bad_r, q), (r, bad_q)):
        d_r = torch.tensor(rr, dtype=torch.float64, device="cuda")
        d_q = torch.tensor(qq, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        with pytest.raises(P.HPDMKError) as e:
            P.HPDMKPtTree(params, None, None, device_inputs=(d_r.data_ptr(), d_q.data_ptr(), n))
        assert e.value.code == 2 and "positions must lie" in str(e.value)
    d_r = torch.tensor(r, dtype=torch.float64, device="cuda")
    d_q = torch.tensor(q, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g = P.HPDMKPtTree(params, None, None, device_inputs=(d_r.data_ptr(), d_q.data_ptr(), n))
    h = P.HPDMKPtTree(params, r, q)
    try:
        for t in (g, h):
            t.form_outgoing_pw()
            t.form_incoming_pw()
        assert g.eval_energy() == h.eval_energy()
    finally:
        g.close()
        h.close()


@pytest.mark.parametrize("case", CASES)
def test_tree_bit_exact(case):
    g, o, r, q = pair(*case)
    assert g.max_depth == o.max_depth and g.n_nodes == o.n_nodes
    for a, b in zip(g.tree_nodes(), o.tree_nodes()):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(g.tree_neighbors(), o.tree_neighbors()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(g.sorted_order(), o.sorted_order())


@pytest.mark.parametrize("case", CASES)
def test_expansions_and_energy(case):
    g, o, r, q = pair(*case)
    np.testing.assert_allclose(g.window_matrix(), o.window_matrix(), rtol=1e-12,
                               atol=1e-14 * np.abs(o.window_matrix()).max())
    for l in range(2, g.max_depth - 1):
        D = o.difference_matrix(l)
        np.testing.assert_allclose(g.difference_matrix(l), D, rtol=1e-12, atol=1e-14 * np.abs(D).max())
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    ro, rg = o.pw(0), g.pw(0)
    assert np.abs(rg - ro).max() <= REL_PW * np.abs(ro).max() + 1e-13
    lv, pf, leaf, cnt = o.tree_nodes()
    for node in np.nonzero((lv >= 2) & (lv <= o.max_depth - 2))[0][:200]:
        a, b = g.pw(node), o.pw(node)
        assert np.abs(a - b).max() <= REL_PW * max(1.0, np.abs(b).max()), node
        if not leaf[node]:
            a, b = g.pw(node, "inc"), o.pw(node, "inc")
            assert np.abs(a - b).max() <= REL_PW * max(1.0, np.abs(b).max()), node
    pg, po = g.eval_energy_parts(), o.eval_energy_parts()
    E = po.sum()
    assert np.all(np.abs(pg - po) <= REL_E * abs(E)), (pg, po)


@pytest.mark.parametrize("case", CASES[:3] + CASES[4:])
def test_shift_and_update_sequence(case):
    g, o, r, q = pair(*case)
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    rng = np.random.default_rng(11)
    n, L = len(q), case[2]
    for step in range(24):
        i = int(rng.integers(0, n))
        d = rng.uniform(-0.5, 0.5, 3) * (L / 10 if step % 3 else L)
        pg = g.eval_shift_energy_parts(i, *d)
        vo, po = o.eval_shift_energy(i, *d, parts=True)
        assert np.all(np.abs(pg - po) <= ABS_DE * max(1.0, np.abs(po).max())), (step, pg, po)
        if step % 2 == 0:
            g.update_shift(i, *d)
            o.update_shift(i, *d)
    np.testing.assert_array_equal(g.positions(), o.positions())
    pg, po = g.eval_energy_parts(), o.eval_energy_parts()
    assert np.all(np.abs(pg - po) <= REL_E * abs(po.sum())), (pg, po)


def test_overflow_pool_and_repack():
    # no slack: every move into another leaf parks the particle in the pool
    g, o, r, q = pair("uniform", 1500, 10.0, 10, 6, slack=0, seed=3)
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    rng = np.random.default_rng(5)
    for step in range(30):
        i = int(rng.integers(0, 1500))
        d = rng.uniform(-2.0, 2.0, 3)
        dg = g.eval_shift_energy(i, *d)
        do = o.eval_shift_energy(i, *d)
        assert abs(dg - do) <= ABS_DE * max(1.0, abs(do)), step
        g.update_shift(i, *d)
        o.update_shift(i, *d)
    np.testing.assert_array_equal(g.positions(), o.positions())
    pg, po = g.eval_energy_parts(), o.eval_energy_parts()
    assert np.all(np.abs(pg - po) <= REL_E * abs(po.sum()))
    # after the repack inside eval_energy, moves keep agreeing
    for step in range(6):
        i = int(rng.integers(0, 1500))
        d = rng.uniform(-1.0, 1.0, 3)
        assert abs(g.eval_shift_energy(i, *d) - o.eval_shift_energy(i, *d)) <= ABS_DE


def test_batch():
    g, o, r, q = pair("uniform", 3000, 14.4, 12, 9, seed=9)
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    rng = np.random.default_rng(2)
    m = 64
    idx = rng.integers(0, 3000, m)
    disp = rng.uniform(-0.5, 0.5, (m, 3))
    dg = g.eval_shift_energy_batch(idx, disp)
    do = np.array([o.eval_shift_energy(i, *d) for i, d in zip(idx, disp)])
    assert np.abs(dg - do).max() <= ABS_DE


METROPOLIS_CASES = [
    ("uniform", 3000, 14.4, 12, 9, 8),
    ("clustered", 4000, 20.0, 10, 6, 0),   # no slack: arrivals go to the overflow pool
    ("uniform", 1500, 10.0, 10, 12, 2),
    ("reference", 1000, 20.0, 10, 3, 4),
]


@pytest.mark.parametrize("mode", [P.MC_PERSISTENT, P.MC_GRAPH])
@pytest.mark.parametrize("case", METROPOLIS_CASES)
def test_metropolis(mode, case):
    # sequential Metropolis: the oracle replays the same proposals. The graph
    # mode runs 300 moves as two captured 128-move graphs plus 44 direct
    # launch pairs; the persistent mode as one cooperative launch.
    kind, n, L, npl, digits, slack = case
    g, o, r, q = pair(kind, n, L, npl, digits, slack=slack, seed=9)
    g.set_mc_mode(mode)
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    rng = np.random.default_rng(2)
    m = 300
    idx = rng.integers(0, n, m)
    disp = rng.uniform(-0.5, 0.5, (m, 3))
    u = rng.uniform(0, 1, m)
    beta = 1.0
    dEg, accg = g.mc_run(idx, disp, u, beta)
    for c in range(m):
        de = o.eval_shift_energy(idx[c], *disp[c])
        assert abs(de - dEg[c]) <= ABS_DE * max(1.0, abs(de)), c
        acc = u[c] < np.exp(-beta * de)
        assert abs(u[c] - np.exp(-beta * de)) < 1e-9 or acc == bool(accg[c])
        if accg[c]:
            o.update_shift(idx[c], *disp[c])
    assert accg.sum() > 0
    np.testing.assert_array_equal(g.positions(), o.positions())
    pg, po = g.eval_energy_parts(), o.eval_energy_parts()
    assert np.all(np.abs(pg - po) <= REL_E * abs(po.sum()))
    # a second run continues from the updated state
    idx = rng.integers(0, n, 40)
    disp = rng.uniform(-0.5, 0.5, (40, 3))
    dg = g.eval_shift_energy_batch(idx, disp)
    do = np.array([o.eval_shift_energy(i, *d) for i, d in zip(idx, disp)])
    assert np.abs(dg - do).max() <= ABS_DE * max(1.0, np.abs(do).max())


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_reference_shift_scenario_vs_ewald(digits):
    # compare_shift_energy / compare_update (test/hpdmk_test.cpp:374-533) on the GPU path
    L, n = 20.0, 1000
    r, q = O.reference_test_system(n, L)
    s = 6.0 if digits == 12 else 5.0
    Eold = O.ewald_energy(L, r, q, s=s, alpha=1.0)
    ew = O.EwaldMC(L, r, q, s=s, alpha=1.0)
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=10, digits=digits, L=L, init=P.DIRECT), r, q)
    g.form_outgoing_pw()
    g.form_incoming_pw()
    E = g.eval_energy()
    assert abs((E - Eold) / Eold) < 5 * 10.0 ** (-digits + 1)
    d, idx = O.reference_trials(10, L, n)
    for k in range(10):
        dE = g.eval_shift_energy(idx[k], *d[k])
        dEe = ew.shift(idx[k], d[k])
        assert abs((dEe - dE) / Eold) < 5 * 10.0 ** (-digits + 1)
        g.update_shift(idx[k], *d[k])
        ew.move(idx[k], d[k])
        assert abs(dEe - dE) < 10.0 ** (-digits + 1)


def test_edge_cases():
    L = 8.0
    # a single charge: the energy is its periodic self-image energy; any move costs nothing
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=4, digits=6, L=L, init=P.DIRECT), np.array([1.0, 2.0, 3.0]),
                      np.array([1.0]))
    o = O.OracleTree(L, 4, 6, np.array([1.0, 2.0, 3.0]), np.array([1.0]))
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    assert abs(g.eval_energy() - o.eval_energy()) <= 1e-12
    assert abs(g.eval_shift_energy(0, 1.5, -2.0, 7.9)) <= 1e-11
    # boundary coordinates, a full-box displacement and a multi-box wrap
    rng = np.random.default_rng(4)
    r = rng.uniform(0, L, (500, 3))
    r[0] = [0.0, 0.0, 0.0]
    r[1] = [np.nextafter(L, 0), np.nextafter(L, 0), 0.0]
    r[2] = [L / 2, L / 4, L / 8]
    q = np.where(np.arange(500) % 2 == 0, 1.0, -1.0)
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=6, digits=9, L=L, init=P.DIRECT), r.reshape(-1), q)
    o = O.OracleTree(L, 6, 9, r.reshape(-1), q)
    for a, b in zip(g.tree_nodes(), o.tree_nodes()):
        np.testing.assert_array_equal(a, b)
    for t in (g, o):
        t.form_outgoing_pw()
        t.form_incoming_pw()
    for i, d in [(0, (L, 0.0, 0.0)), (1, (1e-9, 0.0, -1e-9)), (2, (0.0, 0.0, 0.0)), (3, (-2.5 * L, 3.25 * L, 0.5)),
                 (4, (-1e-300, 0.0, 0.0))]:
        dg, do = g.eval_shift_energy(i, *d), o.eval_shift_energy(i, *d)
        assert abs(dg - do) <= ABS_DE * max(1.0, abs(do)), (i, d, dg, do)
        g.update_shift(i, *d)
        o.update_shift(i, *d)
    np.testing.assert_array_equal(g.positions(), o.positions())
    assert abs(g.eval_energy() - o.eval_energy()) <= REL_E * abs(o.eval_energy())
