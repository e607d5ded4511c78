"""The first configuration, as stated: N = 1000 point charges uniform in a
periodic cube of side L = 10, alternating +1 / -1 charges, 6 digits
(n_per_leaf = 10: with the reference's default of 200 the tree would have
fewer than three levels, which the reference rejects, src/tree.cpp:352).
The full energy, then 100 single-particle energy shifts (a random particle,
a displacement uniform in [-0.5, 0.5]^3, wrapped into the box), each checked
against the oracle's FP64 Ewald (the reference's compare_shift_energy,
test/hpdmk_test.cpp:374-467, tolerance 5 10^(1-d) |E_Ewald|) and against the
oracle's DMK tree, for the FP64 and the mixed-precision path."""
import numpy as np
import pytest

import pdmk4mc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, L, DIGITS, NPL = 1000, 10.0, 6, 10
REL_EWALD = 5 * 10.0 ** (1 - DIGITS)  # the reference's energy and shift tolerance, relative to |E|
REL_E = 1e-11      # FP64 GPU against the FP64 oracle tree
ABS_DE = 2e-10
REL_E_MIXED = 10.0 ** -(DIGITS + 1)  # mixed against the FP64 oracle tree: a tenth of the method's error
ABS_DE_MIXED = 1e-8


def config1():
    rng = np.random.default_rng(2024)
    r = rng.uniform(0, L, 3 * N)
    q = np.where(np.arange(N) % 2 == 0, 1.0, -1.0)
    idx = rng.integers(0, N, 100)
    disp = rng.uniform(-0.5, 0.5, (100, 3))
    return r, q, idx, disp


@pytest.mark.parametrize("precision", [P.PRECISION_FP64, P.PRECISION_MIXED])
def test_config1_energy_and_shifts_vs_ewald(precision):
    r, q, idx, disp = config1()
    ew = O.EwaldMC(L, r, q)
    E_ew = O.ewald_energy(L, r, q)
    o = O.OracleTree(L, NPL, DIGITS, r, q)
    o.form_outgoing_pw()
    o.form_incoming_pw()
    Eo = o.eval_energy()
    g = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=NPL, digits=DIGITS, L=L, init=P.DIRECT), r, q,
                      precision=precision)
    mixed = precision == P.PRECISION_MIXED
    try:
        g.form_outgoing_pw()
        g.form_incoming_pw()
        E = g.eval_energy()
        print(f"\nACCURACY config 1 precision={precision}: vs Ewald {abs(E - E_ew) / abs(E_ew):.3e}, "
              f"vs oracle {abs(E - Eo) / abs(Eo):.3e}")
        assert abs(E - E_ew) <= REL_EWALD * abs(E_ew), (E, E_ew)
        assert abs(E - Eo) <= (REL_E_MIXED if mixed else REL_E) * abs(Eo), (E, Eo)
        dE = np.array([g.eval_shift_energy(int(i), *d) for i, d in zip(idx, disp)])
        dEo = np.array([o.eval_shift_energy(int(i), *d) for i, d in zip(idx, disp)])
        dEw = np.array([ew.shift(int(i), d) for i, d in zip(idx, disp)])
        assert np.all(np.abs(dE - dEw) <= REL_EWALD * abs(E_ew)), np.abs(dE - dEw).max() / abs(E_ew)
        tol = ABS_DE_MIXED if mixed else ABS_DE
        assert np.all(np.abs(dE - dEo) <= tol * np.maximum(1.0, np.abs(dEo))), np.abs(dE - dEo).max()
        # the batched form of the same 100 candidates
        dEb = g.eval_shift_energy_batch(idx, disp)
        assert np.all(np.abs(dEb - dEo) <= tol * np.maximum(1.0, np.abs(dEo)))
    finally:
        g.close()
