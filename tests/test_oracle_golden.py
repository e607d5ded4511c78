"""Pins the oracle (CPU restatement) to the reference: golden vectors made
from the reference's own compiled math (tests/golden/make_golden.py) and the
reference test-suite's known answers and tolerances (test/*.cpp)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import pswf

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_math.npz"))


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_pswf_constants(digits):
    k = pswf.constants(digits)
    assert k["c"] == G[f"d{digits}_c"]
    assert k["n_diff"] == G[f"d{digits}_n_diff"]
    np.testing.assert_array_equal(np.array(k["poly_horner"]), G[f"d{digits}_poly_horner"])
    assert abs(k["lam"] / G[f"d{digits}_lambda"] - 1) < 1e-12
    # psi_0 normalisation is free; compare normalisation-independent ratios
    p0_ref = G[f"d{digits}_psi0"][0]
    assert abs(k["C0"] / k["psi0_0"] - G[f"d{digits}_C0"] / p0_ref) < 1e-13
    assert abs(k["diff0"] / G[f"d{digits}_diff0"] - 1) < 1e-12
    mine = pswf.psi0(k["legendre"], G[f"d{digits}_psi0_x"]) / k["psi0_0"]
    np.testing.assert_allclose(mine, G[f"d{digits}_psi0"] / p0_ref, rtol=0, atol=1e-14)
    # zero outside [-1, 1], as the reference evaluates it for c < 45
    assert np.all(G[f"d{digits}_psi0"][G[f"d{digits}_psi0_x"] > 1] == 0)


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_residual_kernel(digits):
    k = pswf.constants(digits)
    poly = np.ascontiguousarray(k["poly_horner"])
    got = np.array([O.lib().or_res_kernel(len(poly), O._p(poly), r, 0.8) for r in G[f"d{digits}_res_r"]])
    np.testing.assert_allclose(got, G[f"d{digits}_res"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("digits,L", [(3, 20.0), (6, 10.0), (9, 46.4)])
def test_kernel_matrices(digits, L):
    # a deep tree so that levels 2 and 3 both carry difference kernels
    r = O.random_init(3 * 4000, 0.0, L)
    q = np.where(np.arange(4000) % 2 == 0, 1.0, -1.0)
    T = O.OracleTree(L, 4, digits, r, q)
    assert T.max_depth >= 5
    # entries where psi_0 is tiny (k sigma near 1) carry the Legendre tail's
    # cancellation; the bound is relative to the matrix scale
    W = G[f"W_d{digits}_L{L}"]
    np.testing.assert_allclose(T.window_matrix(), W, rtol=1e-11, atol=1e-13 * np.abs(W).max())
    for lvl in (2, 3):
        D = G[f"D{lvl}_d{digits}_L{L}"]
        np.testing.assert_allclose(T.difference_matrix(lvl), D, rtol=1e-11, atol=1e-13 * np.abs(D).max())


def test_shift_phases():
    n, L = 6, 20.0
    for lvl in (2, 3, 4):
        dk = (2 * np.pi / 3) / (L / 2 ** lvl)
        for (px, py, pz) in ((1, 0, 0), (0, -1, 0), (-1, 1, 1), (1, 1, -1)):
            got = np.zeros(2 * (2 * n + 1) ** 2 * (n + 1))
            O.lib().or_shift_phases(n, dk, L, px, py, pz, O._p(got))
            np.testing.assert_allclose(got, G[f"shift_l{lvl}_{px}{py}{pz}"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("N", [13, 25])
def test_nudft_halfplane(N):
    x, y, z = [np.ascontiguousarray(a) for a in G[f"nudft_N{N}_xyz"]]
    q = np.ascontiguousarray(G[f"nudft_N{N}_q"])
    f = np.zeros_like(G[f"nudft_N{N}_f"])
    O.lib().or_nudft_halfplane(len(q), O._p(x), O._p(y), O._p(z), O._p(q), N, O._p(f))
    np.testing.assert_allclose(f, G[f"nudft_N{N}_f"], rtol=0, atol=1e-12)
    g = np.zeros_like(f)
    O.lib().or_nudft_single(x[0], y[0], z[0], q[0], N, O._p(g))
    np.testing.assert_allclose(g, G[f"nudft_single_N{N}_f"], rtol=0, atol=1e-13)
    # and both equal the defining sum e^{-i k.x}, kz <= 0 half space
    n = N // 2
    k = np.arange(N) - n
    kz = np.arange(n + 1) - n
    ph = np.exp(-1j * (kz[:, None, None, None] * z + k[None, :, None, None] * y + k[None, None, :, None] * x))
    direct = (ph * q).sum(-1).reshape(-1)
    got = f[0::2] + 1j * f[1::2]
    np.testing.assert_allclose(got, direct, rtol=0, atol=1e-11)


def test_vecops_formulas():
    A, B, C, W = G["vec_A"], G["vec_B"], G["vec_C"], G["vec_W"]
    a, b, c = A[0::2] + 1j * A[1::2], B[0::2] + 1j * B[1::2], C[0::2] + 1j * C[1::2]
    assert abs(np.sum(np.abs(a) ** 2 * W) - G["vec_doudot"]) < 1e-13
    assert abs(np.sum((a * b).real * W) - G["vec_tridot_nn"]) < 1e-13
    assert abs(np.sum(((a - b) * np.conj(c - b)).real * W) - G["vec_shift_window"]) < 1e-13
    assert abs(np.sum((a * (b - np.conj(a))).real * W) - G["vec_shift_diff_origin"]) < 1e-13
    for add in (0, 1):
        for cj in (0, 1):
            s = 1 if add else -1
            bb = np.conj(b) if cj else b
            exp = a + s * bb
            got = G[f"vec_addsub_{add}{cj}"]
            np.testing.assert_allclose(got[0::2] + 1j * got[1::2], exp, atol=1e-15)
            bc = np.conj(b * c) if cj else b * c
            got = G[f"vec_muladdsub_{add}{cj}"]
            np.testing.assert_allclose(got[0::2] + 1j * got[1::2], a + s * bc, atol=1e-15)


def test_wrap_helpers():
    L = float(G["my_mod_L"])
    got = np.array([O.lib().or_my_mod(v, L) for v in G["my_mod_x"]])
    np.testing.assert_array_equal(got, G["my_mod"])
    got = np.array([O.lib().or_periodic_shift(a, b, L, c, d) for a, b, c, d in G["periodic_shift_cases"]])
    np.testing.assert_array_equal(got, G["periodic_shift"])


def test_random_init_stream():
    np.testing.assert_array_equal(O.random_init(64, 0.0, 20.0), G["random_init_0_20"])


def test_ewald_known_answer():
    ka = json.load(open(os.path.join(HERE, "golden", "ewald_known_answer.json")))
    r = np.array(ka["r"], dtype=np.float64).reshape(-1)
    q = np.array(ka["q"], dtype=np.float64)
    pots = []
    for alpha in ka["alphas"]:
        E = O.ewald_energy(ka["L"], r, q, s=ka["s"], alpha=alpha)
        assert abs(E / (4 * np.pi) - ka["E_over_4pi"]) < ka["tolerance"]
        x, y, z = ka["potential_point"]
        pots.append(O.lib().or_ewald_potential(ka["L"], ka["s"], alpha, len(q), O._p(r), O._p(q), x, y, z, -1, 8))
    assert max(pots) - min(pots) < 1e-10
