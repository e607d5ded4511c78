"""The static-buffer candidate batch (hpdmk_eval_shift_energy_batch_static, no
reference counterpart). It serves callers that may not allocate device memory
once the tree exists: a process whose device memory is handed out up front
(by its own budget or another framework's pool it must not grow), or a
stepping loop that must not enter the allocator, which can synchronise or
fail under fragmentation. The call stages its inputs and outputs in one
fixed static device array and runs the same single launch as the allocating
batch, so its results equal hpdmk_eval_shift_energy_batch bit for bit and
the single-move call hpdmk_eval_shift_energy within the energy-shift
tolerance of the parity tests; on consecutive calls, across two trees that
take turns on the one array, after accepted moves, and with no device
allocation during the calls. Kept in a file that sorts last so it also runs
after every other GPU test."""
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
        for call in range(2):  # two calls in a row through the same static array
            idx, disp = moves(rng, n, 37, 0.4)
            want = t.eval_shift_energy_batch(idx, disp)
            got = t.eval_shift_energy_batch_static(idx, disp)
            np.testing.assert_array_equal(got, want, err_msg=f"call {call}")
            assert np.all(np.isfinite(got))
            for c in range(3):
                close(np.array([t.eval_shift_energy(int(idx[c]), *disp[c])]), got[c:c + 1])
        # the static call changes no tree state: a proposal evaluated before it
        # is still the one update_shift commits
        i0, d0 = moves(rng, n, 1, 0.4)
        before = t.eval_shift_energy(int(i0[0]), *d0[0])
        t.eval_shift_energy_batch_static(*moves(rng, n, 5, 0.4))
        assert t.eval_shift_energy_batch_static(i0, d0)[0] == t.eval_shift_energy_batch(i0, d0)[0]
        close(np.array([before]), t.eval_shift_energy_batch_static(i0, d0))
    finally:
        t.close()


def test_static_batch_two_trees_share_the_array():
    # two trees of different size and digits take turns on the one array
    a, ra = make_tree(2000, 10.0, 10, 6, seed=21)
    b, rb = make_tree(4000, 16.0, 12, 9, seed=22)
    try:
        for turn in range(3):
            for t, rng, n in ((a, ra, 2000), (b, rb, 4000), (a, ra, 2000)):
                idx, disp = moves(rng, n, 64 + 17 * turn, 0.5)
                np.testing.assert_array_equal(t.eval_shift_energy_batch_static(idx, disp),
                                              t.eval_shift_energy_batch(idx, disp))
    finally:
        a.close()
        b.close()


def test_static_batch_after_accepted_moves():
    t, rng = make_tree(2500, 12.0, 10, 9, seed=8)
    try:
        for _ in range(3):
            i, d = moves(rng, 2500, 1, 0.5)
            t.eval_shift_energy(int(i[0]), *d[0])
            t.update_shift(int(i[0]), *d[0])
        idx, disp = moves(rng, 2500, 20, 0.5)
        np.testing.assert_array_equal(t.eval_shift_energy_batch_static(idx, disp), t.eval_shift_energy_batch(idx, disp))
    finally:
        t.close()


def test_static_batch_allocates_nothing():
    # the device's default memory pool (what stream-ordered allocations draw
    # from) must not grow during the calls, not even transiently (its
    # high-water mark is reset first), and the device's free memory must not
    # change (plain allocations)
    from cuda.bindings import driver as dr
    from cuda.bindings import runtime as rt

    def ok(res):
        assert res[0] == rt.cudaError_t.cudaSuccess, res[0]
        return res[1:] if len(res) > 2 else (res[1] if len(res) == 2 else None)

    t, rng = make_tree(3000, 12.0, 10, 9, seed=31)
    try:
        idx, disp = moves(rng, 3000, 64, 0.4)
        t.eval_shift_energy_batch_static(idx, disp)  # first call on the device: finds the array's address
        pool = ok(rt.cudaDeviceGetDefaultMemPool(0))
        used_attr = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent
        high_attr = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
        ok(rt.cudaDeviceSynchronize())
        used0 = int(ok(rt.cudaMemPoolGetAttribute(pool, used_attr)))
        ok(rt.cudaMemPoolSetAttribute(pool, high_attr, dr.cuuint64_t(0)))  # reset to the current use
        free0, _ = ok(rt.cudaMemGetInfo())
        for m in (1, 64, P.STATIC_MAX_MOVES, 300):
            idx, disp = moves(rng, 3000, m, 0.4)
            dE = t.eval_shift_energy_batch_static(idx, disp)
            assert dE.shape == (m,) and np.all(np.isfinite(dE))
        ok(rt.cudaDeviceSynchronize())
        used1 = int(ok(rt.cudaMemPoolGetAttribute(pool, used_attr)))
        high1 = int(ok(rt.cudaMemPoolGetAttribute(pool, high_attr)))
        free1, _ = ok(rt.cudaMemGetInfo())
        # (after its reset the high-water mark reads the current use or, with no
        # allocation event since, zero)
        assert used1 == used0 and high1 <= used0, (used0, used1, high1)
        assert free1 == free0, (free0, free1)
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
        np.testing.assert_array_equal(t.eval_shift_energy_batch_static(idx, disp), t.eval_shift_energy_batch(idx, disp))
    finally:
        t.close()
