"""The reference's own test scenarios (test/hpdmk_test.cpp) run on the
oracle, at the reference's tolerances, plus structural invariants of the
tree the oracle builds (SCTL PtTree semantics)."""
import numpy as np
import pytest

from oracle import oracle as O

L = 20.0


def _ewald_s(digits):
    return 6.0 if digits == 12 else 5.0


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_energy_vs_direct_and_ewald(digits):
    # compare_energy (test/hpdmk_test.cpp:317-372): N = 1000, 1100; n_per_leaf 10
    for i in range(2):
        n = 1000 + 100 * i
        r = O.random_init(3 * n, 0.0, L)
        q = O.random_init(n, -1.0, 1.0)
        q = q - q.sum() / n
        Ee = O.ewald_energy(L, r, q, s=4.0 if digits < 12 else 6.0, alpha=1.0)
        T = O.OracleTree(L, 10, digits, r, q)
        T.form_outgoing_pw()
        T.form_incoming_pw()
        parts = T.eval_energy_parts()
        direct = T.eval_energy_direct_parts()
        tol = 5 * 10.0 ** (-digits + 1)
        assert np.all(np.abs((parts - direct) / Ee) < tol)
        assert abs((parts.sum() - direct.sum()) / Ee) < tol
        # the total against Ewald (the reference's compare uses the direct sums)
        assert abs((parts.sum() - Ee) / Ee) < tol


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_shift_energy_vs_ewald(digits):
    # compare_shift_energy (test/hpdmk_test.cpp:374-467)
    n = 1000
    r, q = O.reference_test_system(n, L)
    s = _ewald_s(digits)
    Eold = O.ewald_energy(L, r, q, s=s, alpha=1.0)
    ew = O.EwaldMC(L, r, q, s=s, alpha=1.0)
    T = O.OracleTree(L, 10, digits, r, q)
    T.form_outgoing_pw()
    T.form_incoming_pw()
    d, idx = O.reference_trials(10, L, n)
    for k in range(10):
        dE = T.eval_shift_energy(idx[k], *d[k])
        dEe = ew.shift(idx[k], d[k])
        assert abs((dEe - dE) / Eold) < 5 * 10.0 ** (-digits + 1)


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_sequential_update_vs_ewald(digits):
    # compare_update (test/hpdmk_test.cpp:470-533)
    n = 1000
    r, q = O.reference_test_system(n, L)
    s = _ewald_s(digits)
    ew = O.EwaldMC(L, r, q, s=s, alpha=1.0)
    T = O.OracleTree(L, 10, digits, r, q)
    T.form_outgoing_pw()
    T.form_incoming_pw()
    d, idx = O.reference_trials(10, L, n)
    for k in range(10):
        dE = T.eval_shift_energy(idx[k], *d[k])
        T.update_shift(idx[k], *d[k])
        dEe = ew.move(idx[k], d[k])
        assert abs(dEe - dE) < 10.0 ** (-digits + 1)
    # the maintained expansions equal a fresh tree's energy on the moved system
    T2 = O.OracleTree(L, 10, digits, T.positions(), q)
    T2.form_outgoing_pw()
    T2.form_incoming_pw()
    assert abs(T.eval_energy() - T2.eval_energy()) < 1e-12 * abs(T2.eval_energy())


def _morton_decode(p):
    x = y = z = 0
    for b in range(21):
        x |= ((p >> (3 * b)) & 1) << b
        y |= ((p >> (3 * b + 1)) & 1) << b
        z |= ((p >> (3 * b + 2)) & 1) << b
    return x, y, z


@pytest.mark.parametrize("case", ["uniform", "clustered"])
def test_tree_invariants(case):
    rng = np.random.default_rng(7)
    n = 6000
    if case == "uniform":
        r = rng.uniform(0, L, (n, 3))
    else:
        c = rng.uniform(0, L, (4, 3))
        r = np.mod(c[rng.integers(0, 4, n)] + rng.normal(0, L / 40, (n, 3)), L)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    T = O.OracleTree(L, 20, 6, r.reshape(-1), q)
    lv, pf, leaf, cnt = T.tree_nodes()
    col, cg = T.tree_neighbors()
    # level-major, Morton within a level, all leaves at level >= 2
    assert np.all(np.diff(lv) >= 0)
    for l in range(T.max_depth):
        assert np.all(np.diff(pf[lv == l].astype(np.int64)) > 0)
    assert np.all(lv[leaf == 1] >= 2)
    # counts: leaves hold at most n_per_leaf unless at the depth cap
    assert np.all(cnt[(leaf == 1) & (lv < 10)] <= 20)
    assert cnt[0] == n
    # every non-leaf node at level >= 2 has 26 colleagues (src/planewave.cpp:130)
    nl = (leaf == 0) & (lv >= 2)
    assert np.all((col[nl] >= 0).sum(1) == 26)
    # 2:1 balance: a leaf's neighbouring regions are covered by leaves at most one level apart
    keyset = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lv, pf))}
    for i in np.nonzero(leaf)[0]:
        l = int(lv[i])
        x, y, z = _morton_decode(int(pf[i]))
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    m = (1 << l) - 1
                    nx, ny, nz = (x + dx) & m, (y + dy) & m, (z + dz) & m
                    # the deepest existing ancestor-or-self of the neighbour cell
                    found = None
                    for ll in range(l, -1, -1):
                        sh = l - ll
                        a, b, c2 = nx >> sh, ny >> sh, nz >> sh
                        pfx = 0
                        for bit in range(ll):
                            pfx |= ((a >> bit) & 1) << (3 * bit) | ((b >> bit) & 1) << (3 * bit + 1) | ((c2 >> bit) & 1) << (3 * bit + 2)
                        if (ll, pfx) in keyset:
                            found = keyset[(ll, pfx)]
                            break
                    # checked from the finer side of every adjacent leaf pair
                    assert found is not None
                    if leaf[found]:
                        assert l - lv[found] <= 1
    # leaf paths contain the point (test/hpdmk_test.cpp:262-265)
    for k in range(50):
        pt = rng.uniform(0, L, 3)
        path = T.leaf_path(*pt)
        assert leaf[path[-1]] == 1 and path[0] == 0
        for depth, node in enumerate(path):
            x, y, z = _morton_decode(int(pf[node]))
            bs = L / 2 ** lv[node]
            assert lv[node] == depth
            for coord, ic in zip(pt, (x, y, z)):
                assert ic * bs <= coord < (ic + 1) * bs
