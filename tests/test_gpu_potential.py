"""Potentials and fields (hpdmk_eval_potential, phi_i = dE/dq_i): the energy
is 1/2 sum q_i phi_i; differences of potentials between equal charges match
the oracle's FP64 Ewald potential of all other particles (the charge-
proportional self-image and background terms cancel in them); the field
matches central differences of the Ewald potential."""
import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

def make(n, L, digits, npl, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT), r, q, leaf_slack=4)
    t.form_outgoing_pw()
    t.form_incoming_pw()
    return t, r, q, rng


@pytest.mark.parametrize("digits", [6, 9, 12])
def test_potential_vs_ewald(digits):
    n, L = 2000, 12.6
    t, r, q, rng = make(n, L, digits, 10, digits)
    try:
        idx = rng.choice(np.arange(0, n, 2), 24, replace=False)  # charge +1
        phi, field = t.potential(idx)
        s = 4.0 if digits < 12 else 6.0
        ref = np.array([O.ewald_potential(L, r, q, int(i), r[3 * i:3 * i + 3], s=s) for i in idx])
        # pointwise potentials carry the method's error without the averaging an
        # energy sum gets: 10^(2-d) of their scale
        dd, de = phi - phi[0], ref - ref[0]
        assert np.all(np.abs(dd - de) <= 10.0 ** (2 - digits) * np.maximum(1.0, np.abs(de))), (digits, dd - de)
        if digits >= 9:
            def cd(x, i, a, h):  # central difference of -phi along axis a
                e = np.zeros(3)
                e[a] = h
                return -(O.ewald_potential(L, r, q, int(i), np.mod(x + e, L), s=s) -
                         O.ewald_potential(L, r, q, int(i), np.mod(x - e, L), s=s)) / (2 * h)
            for c, i in enumerate(idx[:8]):
                x = r[3 * i:3 * i + 3]
                for a in range(3):
                    fd = (4 * cd(x, i, a, 1e-3) - cd(x, i, a, 2e-3)) / 3  # Richardson: O(h^4)
                    # a derivative carries more of the method's error (about 1e-6 at
                    # 9 digits); the difference quotient itself is good to about 1e-7
                    tol = max(10.0 ** (4 - digits), 1e-6)
                    assert abs(field[c, a] - fd) <= tol * max(1.0, abs(fd)), (i, a, field[c, a], fd)
    finally:
        t.close()


@pytest.mark.parametrize("digits", [6, 9])
def test_energy_is_half_sum_q_phi(digits):
    n, L = 3000, 14.4
    t, r, q, _ = make(n, L, digits, 12, digits)
    try:
        phi = t.potential(np.arange(n), field=False)
        e = t.eval_energy()
        assert abs(e - 0.5 * np.dot(q, phi)) <= 1e-11 * abs(e), (e, 0.5 * np.dot(q, phi))
    finally:
        t.close()


def test_potential_follows_moves():
    n, L = 2500, 13.6
    t, r, q, rng = make(n, L, 9, 12, 7)
    try:
        for _ in range(40):
            i = int(rng.integers(0, n))
            d = rng.uniform(-0.5, 0.5, 3)
            t.eval_shift_energy(i, *d)
            t.update_shift(i, *d)
        pos = np.ascontiguousarray(t.positions())
        idx = rng.choice(np.arange(1, n, 2), 12, replace=False)  # charge -1
        phi = t.potential(idx, field=False)
        ref = np.array([O.ewald_potential(L, pos, q, int(i), pos[3 * i:3 * i + 3]) for i in idx])
        assert np.all(np.abs((phi - phi[0]) - (ref - ref[0])) <= 1e-8 * np.maximum(1.0, np.abs(ref - ref[0])))
    finally:
        t.close()
