"""CPU checks of the two precision decisions of the mixed path, restated in
numpy on the same inputs the kernels see.

1. The outgoing expansion of one box from 8-bit slices: the kernel's
   arithmetic (FP32 phase factors, t = 127 v split as t = a1 + a2/254 +
   a3/254^2, the six slice products summed exactly in integers, FP64
   combination) against the FP64 direct NUDFT of the reference
   (include/nudft.hpp:95-121). The coefficient error stays near the FP32
   rounding of the operands.
2. The near field in FP32 (box-centred coordinates, FP32 distance and the
   19-term residual polynomial in FP32) misses the 1e-8 energy target on the
   N = 1e5 cube, which is why the near field stays FP64 in both paths.
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


def slices(t):
    """t (float32, |t| <= 127) -> int8 slices a1, a2, a3 with t ~ a1 + a2/254 + a3/254^2."""
    t = t.astype(np.float64)
    a1 = np.rint(t)
    r1 = t - a1
    a2 = np.rint(f32(r1 * 254.0).astype(np.float64))
    r2 = f32(r1 * 254.0 - a2).astype(np.float64)
    a3 = np.rint(f32(r2 * 254.0).astype(np.float64))
    return [a.astype(np.int64) for a in (a1, a2, a3)]


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
    # the kernel: FP32 factors (ex scaled by 127, ez by 127 q / max|q|), A = ez ey in FP32
    qmax = np.abs(q).max()
    exs = f32(127 * ex.real) + 1j * f32(127 * ex.imag)
    eys = f32(ey.real) + 1j * f32(ey.imag)
    ezs = f32(127 * ez.real / qmax) + 1j * f32(127 * ez.imag / qmax)
    A = ezs[:, :, None] * eys[:, None, :]  # [j, kz, ky], products of FP32 values
    Ar, Ai = f32(A.real), f32(A.imag)
    Br, Bi = f32(exs.real), f32(exs.imag)
    sa_r, sa_i, sb_r, sb_i = slices(Ar), slices(Ai), slices(Br), slices(Bi)
    acc_re = [0, 0, 0]
    acc_im = [0, 0, 0]
    for s in range(3):
        for t in range(3 - s):
            # real output: Ar Br - Ai Bi; imaginary: Ar Bi + Ai Br (exact integers)
            acc_re[s + t] = acc_re[s + t] + np.einsum("jzy,jx->zyx", sa_r[s], sb_r[t]) - \
                np.einsum("jzy,jx->zyx", sa_i[s], sb_i[t])
            acc_im[s + t] = acc_im[s + t] + np.einsum("jzy,jx->zyx", sa_r[s], sb_i[t]) + \
                np.einsum("jzy,jx->zyx", sa_i[s], sb_r[t])
    scale = qmax / (127.0 * 127.0)
    out = scale * ((acc_re[0] + acc_re[1] / 254.0 + acc_re[2] / 254.0 ** 2) +
                   1j * (acc_im[0] + acc_im[1] / 254.0 + acc_im[2] / 254.0 ** 2))
    err = np.abs(out - ref).max() / np.abs(ref).max()
    rms = np.sqrt(np.mean(np.abs(out - ref) ** 2)) / np.sqrt(n_box)
    print(f"\nint8 slices, one box of {n_box}: max error {err:.2e} of the largest coefficient, "
          f"rms error per sqrt(particle) {rms:.2e}")
    assert err < 1e-6
    assert rms < 2e-7  # about the FP32 rounding of the operands


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
    print(f"\nFP32 near field on the N=1e5 cube: {len(pairs)} pairs, energy error {rel:.2e} of |E|")
    assert rel > 1e-8
