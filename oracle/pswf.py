"""ORACLE — test infrastructure only.

numpy restatement of the reference's prolate spheroidal wave function
machinery (src/pswf.cpp) and of get_prolate_params (include/utils.hpp:20-52):

* psi_0^c on [-1, 1] is the even Legendre series whose coefficients are the
  eigenvector of the smallest eigenvalue of the prolate differential operator
  -(1-x^2)d^2/dx^2 + 2x d/dx + c^2 x^2 written in the normalised Legendre
  basis (the reference solves the same tridiagonal problem, prolmatr /
  prolql1 / prolsolv, src/pswf.cpp:635-845);
* outside [-1, 1] psi_0^c is zero, as the reference's prol0eva returns for
  every c below its threshold 45 (src/pswf.cpp:976-982);
* lambda = int_{-1}^{1} psi(x) cos(c x / 2) dx / psi(1/2) with 200 Gauss nodes
  (prolate0_lambda, src/pswf.cpp:1208-1218); C0 = int_0^1 psi and
  int_0^1 x^2 psi with 200 Gauss nodes on [0, r] (prol0int0r / prol0x2int0r,
  src/pswf.cpp:997-1058).

Only ratios psi/C0 and lambda enter the method, so the normalisation of psi
is irrelevant; psi(0) > 0 is chosen.
"""
from __future__ import annotations

import numpy as np
from numpy.polynomial import legendre as npleg

# The reference's accuracy table (include/utils.hpp:20-52): bandwidth c,
# difference-kernel mode count n_diff and the residual-kernel polynomial in
# ascending powers of x_scaled = 2 r / b - 1.
PROLATE_TABLE = {
    3: (7.2462000846862793, 6, [
        1.627823522210361e-01, -4.553645597616490e-01, 4.171687104204163e-01, -7.073638602709915e-02,
        -8.957845614474928e-02, 2.617986644718201e-02, 9.633427876507601e-03]),
    6: (13.739999771118164, 12, [
        5.482525801351582e-02, -2.616592110444692e-01, 4.862652666337138e-01, -3.894296348642919e-01,
        1.638587821812791e-02, 1.870328434198821e-01, -8.714171086568978e-02, -3.927020727017803e-02,
        3.728187607052319e-02, 3.153734425831139e-03, -8.651313377285847e-03, 1.725110090795567e-04,
        1.034762385284044e-03]),
    9: (20.736000061035156, 19, [
        1.835718730962269e-02, -1.258015846164503e-01, 3.609487248584408e-01, -5.314579651112283e-01,
        3.447559412892380e-01, 9.664692318551721e-02, -3.124274531849053e-01, 1.322460720579388e-01,
        9.773007866584822e-02, -1.021958831082768e-01, -3.812847450976566e-03, 3.858117355875043e-02,
        -8.728545924521301e-03, -9.401196355382909e-03, 4.024549377076924e-03, 1.512806105865091e-03,
        -9.576734877247042e-04, -1.303457547418901e-04, 1.100385844683190e-04]),
    12: (27.870000839233398, 26, [
        6.262472576363448e-03, -5.605742936112479e-02, 2.185890864792949e-01, -4.717350304955679e-01,
        5.669680214206270e-01, -2.511606878849214e-01, -2.744523658778361e-01, 4.582527599363415e-01,
        -1.397724810121539e-01, -2.131762135835757e-01, 1.995489373508990e-01, 1.793390341864239e-02,
        -1.035055132403432e-01, 3.035606831075176e-02, 3.153931762550532e-02, -2.033178627450288e-02,
        -5.406682731236552e-03, 7.543645573618463e-03, 1.437788047407851e-05, -1.928370882351732e-03,
        2.891658777328665e-04, 3.332996162099811e-04, -8.397699195938912e-05, -3.015837377517983e-05,
        9.640642701924662e-06]),
}


def legendre_coeffs(c: float) -> np.ndarray:
    """Legendre-series coefficients (all orders, odd ones zero) of psi_0^c."""
    m = int(2 * c) + 60  # even orders 0, 2, ..., 2(m-1); the tail decays super-exponentially
    k = 2.0 * np.arange(m)
    # x^2 P_k = a_k P_{k+2} + b_k P_k + c_k P_{k-2}
    b = ((k + 1) ** 2 / (2 * k + 3) + k ** 2 / (2 * k - 1)) / (2 * k + 1)
    diag = k * (k + 1) + c * c * b
    kp = k[1:]  # k >= 2 couples to k - 2; symmetric form in P_k * sqrt(k + 1/2)
    off = c * c * kp * (kp - 1) / ((2 * kp - 1) * np.sqrt((2 * kp - 3) * (2 * kp + 1)))
    A = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    w, v = np.linalg.eigh(A)
    beta = v[:, np.argmin(w)]
    alpha = beta * np.sqrt(k + 0.5)
    coef = np.zeros(2 * m)
    coef[0::2] = alpha
    if npleg.legval(0.0, coef) < 0:
        coef = -coef
    return coef


def psi0(coef: np.ndarray, x):
    x = np.asarray(x, dtype=np.float64)
    val = npleg.legval(np.clip(x, -1.0, 1.0), coef)
    return np.where(np.abs(x) > 1.0, 0.0, val)


def _gauss01(npts: int = 200):
    x, w = npleg.leggauss(npts)
    return x, w


def constants(digits: int) -> dict:
    """Set-up constants of form_wavenumbers (src/tree.cpp:17-81)."""
    if digits not in PROLATE_TABLE:
        raise ValueError("double only supports 3, 6, 9 and 12 digits accuracy")
    c, n_diff, asc = PROLATE_TABLE[digits]
    coef = legendre_coeffs(c)
    xg, wg = _gauss01(200)
    lam = float(np.sum(wg * psi0(coef, xg) * np.cos(c * xg * 0.5)) / psi0(coef, 0.5))
    xs = (xg + 1) * 0.5
    C0 = float(np.sum(wg * 0.5 * psi0(coef, xs)))
    intx2 = float(np.sum(wg * 0.5 * psi0(coef, xs) * xs * xs))
    diff0 = -2.0 * np.pi * intx2 / C0 * c * c
    return dict(digits=digits, c=c, n_diff=n_diff, n_window=int(np.floor(2 * c / np.pi)),
                poly_horner=list(reversed(asc)), legendre=coef, lam=lam, C0=C0, intx2=intx2,
                diff0=diff0, psi0_0=float(psi0(coef, 0.0)))
