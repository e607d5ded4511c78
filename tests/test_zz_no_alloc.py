"""The static-buffer candidate batch (hpdmk_eval_shift_energy_batch_static, no
reference counterpart; it serves callers that may not allocate device memory
after the tree exists, such as a process with a fixed device-memory budget)
against the allocating entry points: the one-block-per-candidate batch
(hpdmk_eval_shift_energy_batch) within the energy-shift tolerance of the
parity tests, and the single-move call (hpdmk_eval_shift_energy, the same
kernel with the same fixed-order reductions) exactly; on consecutive calls
and across trees that share the one static buffer. Kept in a file that sorts
last so it also runs after every other GPU test."""
import numpy as np
import pytest

import pdmk4mc_b200 as P

pytestmark = pytest.mark.gpu

ABS_DE = 2e-10  # energy shifts, absolute (as in the parity tests)


def close(got, want, msg=""):
    np.testing.assert_array_less(np.abs(got - want), ABS_DE * np.maximum(1.0, np.abs(want)), err_msg=msg)


def make_tree(n, L, npl, digits, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=npl, digits=digits, L=L, init=P.DIRECT), r, q)
    t.form_outgoing_pw()
    t.form_incoming_pw()
    t.eval_energy()
    return t, rng


def moves(rng, n, m, step):
    return rng.integers(0, n, m), rng.uniform(-step, step, (m, 3))


@pytest.mark.parametrize("n,L,npl,digits", [(2000, 10.0, 10, 6), (3000, 46.4, 8, 12)])
def test_static_batch_matches_allocating_batch(n, L, npl, digits):
    t, rng = make_tree(n, L, npl, digits, seed=5)
    try:
        for call in range(2):  # two calls in a row through the same static buffer
            idx, disp = moves(rng, n, 37, 0.4)
            want = t.eval_shift_energy_batch(idx, disp)
            got = t.eval_shift_energy_batch_static(idx, disp)
            close(got, want, f"call {call}")
            assert np.all(np.isfinite(got))
            for c in range(3):
                assert t.eval_shift_energy(int(idx[c]), *disp[c]) == got[c]
        # the static call changes no tree state
        i0, d0 = moves(rng, n, 1, 0.4)
        s_static = t.eval_shift_energy_batch_static(i0, d0)[0]
        assert t.eval_shift_energy(int(i0[0]), *d0[0]) == s_static
    finally:
        t.close()


def test_static_batch_after_accepted_moves():
    t, rng = make_tree(2500, 12.0, 10, 9, seed=8)
    try:
        for _ in range(3):
            i, d = moves(rng, 2500, 1, 0.5)
            t.eval_shift_energy(int(i[0]), *d[0])
            t.update_shift(int(i[0]), *d[0])
        idx, disp = moves(rng, 2500, 20, 0.5)
        close(t.eval_shift_energy_batch_static(idx, disp), t.eval_shift_energy_batch(idx, disp))
    finally:
        t.close()


def test_static_batch_rejects_oversize_and_bad_input():
    t, rng = make_tree(500, 8.0, 10, 3, seed=2)
    try:
        m = P.STATIC_MAX_MOVES + 1
        idx, disp = moves(rng, 500, m, 0.3)
        with pytest.raises(P.HPDMKError) as e:
            t.eval_shift_energy_batch_static(idx, disp)
        assert e.value.code == 2 and "static buffer limit" in str(e.value)
        with pytest.raises(P.HPDMKError) as e:
            t.eval_shift_energy_batch_static(np.array([500]), np.zeros((1, 3)))
        assert e.value.code == 2
        assert t.eval_shift_energy_batch_static(np.zeros(0, np.int64), np.zeros((0, 3))).size == 0
        # the largest accepted batch still runs
        idx, disp = moves(rng, 500, P.STATIC_MAX_MOVES, 0.3)
        close(t.eval_shift_energy_batch_static(idx, disp), t.eval_shift_energy_batch(idx, disp))
    finally:
        t.close()
