"""CPU checks of the two precision decisions of the mixed path, restated in
numpy on the same inputs the kernels see.

1. The outgoing expansion of one box from 8-bit slices: the kernel's
   arithmetic (FP64 phase factors, the 32-bit fixed point X = round(127 v
   2^24) (for A each component rounded in two steps, as the kernel's two
   FMAs do: the second term to an integer, then the sum) written as four
   signed base-256 digits, the ten slice products of
   order s + t <= 5 summed exactly in integers, FP64 combination) against the FP64
   direct NUDFT of the reference (include/nudft.hpp:95-121). The
   coefficient error stays near 1e-9 of the largest coefficient.
2. The near field in FP32 (box-centred coordinates, FP32 distance and the
   19-term residual polynomial in FP32) misses the 1e-8 energy target on the
   N = 1e5 cube. With the pair difference and the distance kept in FP64 and
   only the polynomial in FP32 the error is still near half the target, and
   a compensated FP32 Horner scheme (error-free products and sums per term)
   costs more FP32 operations per pair than the FP64 Horner costs FP64 ones
   at the B200's 2:1 FP32:FP64 rate, which is why the near field stays FP64
   in both paths.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import pswf  # noqa: E402


def f32(x):
    return np.asarray(x, dtype=np.float32)


def digits(X):
    """X (a 32-bit fixed point, |X| <= 127 2^24) -> its signed base-256
    digits, highest first, X = sum_s a_s 256^(3-s), every a_s in [-128, 127]:
    the bytes of X + 0x808080, the three lower ones less 128."""
    Y = np.asarray(X).astype(np.int64) + 0x808080
    top = Y >> 24  # arithmetic shift: the signed top digit
    return [top, ((Y >> 16) & 0xFF) - 128, ((Y >> 8) & 0xFF) - 128, (Y & 0xFF) - 128]


def slices(t):
    """t (|t| <= 127) -> the digits of X = round(t 2^24)."""
    return digits(np.rint(t * 2.0 ** 24))


def slices_two_step(z, y):
    """The digits of A = z y's components as the kernel forms them, z already
    carrying 2^24: Re = round(round(-z.im y.im) + z.re y.re) and Im =
    round(round(z.im y.re) + z.re y.im) (each FMA rounds to an integer; the
    products here are rounded to FP64 first, which differs from the fused
    product only within 2^-22 of a half-integer)."""
    re = np.rint(np.rint(-z.imag * y.imag) + z.real * y.real)
    im = np.rint(np.rint(z.imag * y.real) + z.real * y.imag)
    return digits(re), digits(im)


def test_int8_slice_contraction_of_one_box():
    rng = np.random.default_rng(3)
    n_box, nk = 1562, 19  # a level-2 box of the N = 1e5 cube at 9 digits
    bs = 46.4 / 4
    dk = (2 * np.pi / 3) / bs
    x = rng.uniform(-bs / 2, bs / 2, (n_box, 3))
    q = np.where(np.arange(n_box) % 2 == 0, 1.0, -1.0)
    m = np.arange(-nk, nk + 1)
    mz = np.arange(-nk, 1)
    ex = np.exp(-1j * dk * np.outer(x[:, 0], m))
    ey = np.exp(-1j * dk * np.outer(x[:, 1], m))
    ez = np.exp(-1j * dk * np.outer(x[:, 2], mz)) * q[:, None]
    # FP64 reference: out[kz, ky, kx] = sum_j ez ey ex
    ref = np.einsum("jz,jy,jx->zyx", ez, ey, ex)
    # the kernel: FP64 factors (ex scaled by 127, ez by 127 q / max|q|), A = ez ey in FP64
    qmax = np.abs(q).max()
    z = (127 * 2.0 ** 24 * ez / qmax)[:, :, None]  # [j, kz, 1]
    B = 127 * ex
    sa_r, sa_i = slices_two_step(z, ey[:, None, :])  # [j, kz, ky]
    sb_r, sb_i = slices(B.real), slices(B.imag)
    acc_re = [0, 0, 0, 0]
    acc_im = [0, 0, 0, 0]
    for s in range(4):
        for t in range(4 - s):
            # real output: Ar Br - Ai Bi; imaginary: Ar Bi + Ai Br (exact integers)
            acc_re[s + t] = acc_re[s + t] + np.einsum("jzy,jx->zyx", sa_r[s], sb_r[t]) - \
                np.einsum("jzy,jx->zyx", sa_i[s], sb_i[t])
            acc_im[s + t] = acc_im[s + t] + np.einsum("jzy,jx->zyx", sa_r[s], sb_i[t]) + \
                np.einsum("jzy,jx->zyx", sa_i[s], sb_r[t])
    scale = qmax / (127.0 * 127.0)
    w = [256.0 ** -k for k in range(4)]
    out = scale * (sum(a * c for a, c in zip(acc_re, w)) + 1j * sum(a * c for a, c in zip(acc_im, w)))
    # the digits are signed bytes with top digits in [-127, 127], so the exact
    # integer sums fit 32 bits for a split-K chunk of 16384 particles: at most
    # four products per accumulator and K entry, two K entries per particle
    assert all(np.abs(a).max() <= 128 for a in sa_r + sa_i + sb_r + sb_i)
    assert all(np.abs(a[0]).max() <= 127 for a in (sa_r, sa_i, sb_r, sb_i))
    assert 2 * 16384 * (2 * 127 * 128 + 2 * 128 * 128) < 2 ** 31
    assert max(np.abs(a).max() for a in acc_re + acc_im) * 16384 / n_box < 2 ** 31
    err = np.abs(out - ref).max() / np.abs(ref).max()
    rms = np.sqrt(np.mean(np.abs(out - ref) ** 2)) / np.sqrt(n_box)
    print(f"\nint8 slices, one box of {n_box}: max error {err:.2e} of the largest coefficient, "
          f"rms error per sqrt(particle) {rms:.2e}")
    assert err < 2e-9
    assert rms < 2e-9


def test_fp32_near_field_misses_the_target():
    cKDTree = pytest.importorskip("scipy.spatial").cKDTree
    import bench
    W = bench.WORKLOAD_N1E5
    r, q = bench.make_system(1, W["N"], W["L"])
    x = r.reshape(-1, 3)
    L = W["L"]
    ph = np.array(pswf.constants(9)["poly_horner"])
    b = L / 16  # the leaf level of the cube
    pairs = cKDTree(x, boxsize=L).query_pairs(b, output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    d = x[i] - x[j]
    d -= L * np.round(d / L)

    def horner(c, v, dt):
        acc = np.zeros_like(v, dtype=dt)
        for cc in c:
            acc = (acc * v + dt(cc)).astype(dt)
        return acc
    r64 = np.sqrt((d * d).sum(1))
    e64 = np.sum(q[i] * q[j] * horner(ph, (r64 / b - 0.5) * 2, np.float64) / r64)
    cell = (np.floor(x[i] / b) + 0.5) * b  # box-centred FP32 coordinates
    d32 = f32(x[i] - cell) - f32(x[i] - d - cell)
    r32 = np.sqrt((d32 * d32).sum(1, dtype=np.float32)).astype(np.float32)
    x32 = ((r32 * np.float32(1 / b) - np.float32(0.5)) * np.float32(2)).astype(np.float32)
    e32 = np.sum(q[i] * q[j] * (horner(ph.astype(np.float32), x32, np.float32) / r32).astype(np.float64))
    E_total = -7089.02  # the cube's energy (its stored Ewald value)
    rel = abs(e32 - e64) / abs(E_total)
    # FP64 difference and distance, FP32 polynomial only
    xb = ((r64 / b - 0.5) * 2).astype(np.float32)
    ep = np.sum(q[i] * q[j] * horner(ph.astype(np.float32), xb, np.float32).astype(np.float64) / r64)
    rel_poly = abs(ep - e64) / abs(E_total)
    print(f"\nFP32 near field on the N=1e5 cube: {len(pairs)} pairs, energy error {rel:.2e} of |E|; "
          f"FP32 polynomial alone {rel_poly:.2e}")
    assert rel > 1e-8
    assert 2e-9 < rel_poly < 1e-8
