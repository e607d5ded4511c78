"""Generate the golden fixtures that pin the oracle to the reference.

Run in the build container, where the reference sources exist:

    make -C oracle            # builds oracle/_ref/libhpdmk_ref.so from the reference's own
                              # src/pswf.cpp and include/*.hpp (through oracle/ref_shim)
    python tests/golden/make_golden.py

It evaluates the reference's own math (PSWF functions, the accuracy table,
window/difference kernel matrices, shift phases, half-plane NUDFTs, vector
reductions, residual kernel, wrap helpers, the random_init stream) on fixed
inputs and writes tests/golden/reference_math.npz. It also reads the Ewald
known-answer case of test/ewald_test.cpp (100 charges in L=100 and the
EwaldSummations.jl energy) as text and writes tests/golden/ewald_known_answer.json.
"""
from __future__ import annotations

import ctypes
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("HPDMK_REFERENCE", "/root/reference")

dp = ctypes.POINTER(ctypes.c_double)


def P(a):
    return a.ctypes.data_as(dp)


def load_ref():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libhpdmk_ref.so"))
    d = ctypes.c_double
    for f in ("ref_prolate0_eval", "ref_prolate0_int_eval", "ref_prolate0_intx2_eval", "ref_diff0", "ref_my_mod"):
        getattr(L, f).restype = d
        getattr(L, f).argtypes = [d, d]
    L.ref_prolate0_lambda.restype = d
    L.ref_prolate0_lambda.argtypes = [d]
    L.ref_get_prolate_params.restype = ctypes.c_int
    L.ref_get_prolate_params.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.POINTER(ctypes.c_int), dp]
    L.ref_window_matrix.argtypes = [d, d, d, d, d, ctypes.c_int, dp]
    L.ref_difference_matrix.argtypes = [d, d, d, d, d, d, d, ctypes.c_int, dp]
    L.ref_shift_vec.argtypes = [ctypes.c_int, d, d, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    L.ref_nudft3d1_halfplane.argtypes = [ctypes.c_int, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, dp]
    L.ref_nudft3d1_single_halfplane.argtypes = [d, d, d, d, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    for f in ("ref_vec_doudot",):
        getattr(L, f).restype = d
        getattr(L, f).argtypes = [ctypes.c_int, dp, dp]
    L.ref_vec_tridot_nn.restype = d
    L.ref_vec_tridot_nn.argtypes = [ctypes.c_int, dp, dp, dp]
    L.ref_vec_shift_window.restype = d
    L.ref_vec_shift_window.argtypes = [ctypes.c_int, dp, dp, dp, dp]
    L.ref_vec_shift_diff_origin.restype = d
    L.ref_vec_shift_diff_origin.argtypes = [ctypes.c_int, dp, dp, dp]
    L.ref_vec_addsub.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
    L.ref_vec_muladdsub.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ctypes.c_int]
    L.ref_periodic_shift.restype = ctypes.c_int
    L.ref_periodic_shift.argtypes = [d] * 5
    L.ref_residual_kernel.restype = d
    L.ref_residual_kernel.argtypes = [d, ctypes.c_int, d]
    L.ref_random_init.argtypes = [ctypes.c_long, d, d, dp]
    return L


def main():
    R = load_ref()
    out = {}
    rng = np.random.default_rng(20251203)
    # accuracy table and PSWF functions (include/utils.hpp:20-52, src/pswf.cpp)
    xs = np.linspace(0.0, 1.2, 49)
    for dg in (3, 6, 9, 12):
        c, lam, C0 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        nd = ctypes.c_int()
        co = np.zeros(32)
        nco = R.ref_get_prolate_params(dg, ctypes.byref(c), ctypes.byref(lam), ctypes.byref(C0), ctypes.byref(nd), P(co))
        out[f"d{dg}_c"] = c.value
        out[f"d{dg}_lambda"] = lam.value
        out[f"d{dg}_C0"] = C0.value
        out[f"d{dg}_n_diff"] = nd.value
        out[f"d{dg}_poly_horner"] = co[:nco].copy()
        out[f"d{dg}_psi0_x"] = xs
        out[f"d{dg}_psi0"] = np.array([R.ref_prolate0_eval(c.value, x) for x in xs])
        out[f"d{dg}_int_r"] = np.array([0.25, 0.5, 0.75, 1.0])
        out[f"d{dg}_int"] = np.array([R.ref_prolate0_int_eval(c.value, r) for r in out[f"d{dg}_int_r"]])
        out[f"d{dg}_intx2_1"] = R.ref_prolate0_intx2_eval(c.value, 1.0)
        out[f"d{dg}_diff0"] = R.ref_diff0(c.value, C0.value)
        rr = np.linspace(0.0, 0.85, 35)
        out[f"d{dg}_res_r"] = rr
        out[f"d{dg}_res"] = np.array([R.ref_residual_kernel(r, dg, 0.8) for r in rr])
    # k-space kernel matrices (include/kernels.hpp:60-114) as formed in
    # form_interaction_matrices (src/tree.cpp:84-100) for trees of 5 levels
    for dg, L in ((3, 20.0), (6, 10.0), (9, 46.4)):
        c, lam, C0, nd = out[f"d{dg}_c"], out[f"d{dg}_lambda"], out[f"d{dg}_C0"], out[f"d{dg}_n_diff"]
        nw = int(np.floor(2 * c / np.pi))
        sig = [L / c / 2 ** i for i in range(7)]
        bs = [L / 2 ** i for i in range(7)]
        w = np.zeros((2 * nw + 1) ** 2 * (nw + 1))
        R.ref_window_matrix(lam, C0, c, sig[2], 2 * np.pi / L, nw, P(w))
        out[f"W_d{dg}_L{L}"] = w
        diff0 = out[f"d{dg}_diff0"]
        for lvl in (2, 3):
            dmat = np.zeros((2 * nd + 1) ** 2 * (nd + 1))
            R.ref_difference_matrix(lam, C0, c, diff0, sig[lvl], sig[lvl + 1], (2 * np.pi / 3) / bs[lvl], nd, P(dmat))
            out[f"D{lvl}_d{dg}_L{L}"] = dmat
    # shift phases (include/shiftmat.hpp:16-38), half-space part
    for lvl in (2, 3, 4):
        n, L = 6, 20.0
        dk = (2 * np.pi / 3) / (L / 2 ** lvl)
        dd = 2 * n + 1
        for (px, py, pz) in ((1, 0, 0), (0, -1, 0), (-1, 1, 1), (1, 1, -1)):
            v = np.zeros(2 * dd ** 3)
            R.ref_shift_vec(n, dk, L, px, py, pz, P(v))
            out[f"shift_l{lvl}_{px}{py}{pz}"] = v[:2 * dd * dd * (n + 1)]
    # half-plane NUDFT and single-particle NUDFT (include/nudft.hpp:66-167)
    for N in (13, 25):
        M = 37
        x, y, z = (rng.uniform(-9, 9, M) for _ in range(3))
        cq = np.zeros(2 * M)
        cq[0::2] = rng.uniform(-1, 1, M)
        f = np.zeros(2 * N * N * (N // 2 + 1))
        R.ref_nudft3d1_halfplane(M, P(x), P(y), P(z), P(cq), -1, N, N, N, P(f))
        out[f"nudft_N{N}_xyz"] = np.stack([x, y, z])
        out[f"nudft_N{N}_q"] = cq[0::2].copy()
        out[f"nudft_N{N}_f"] = f
        g = np.zeros_like(f)
        R.ref_nudft3d1_single_halfplane(x[0], y[0], z[0], cq[0], -1, N, N, N, P(g))
        out[f"nudft_single_N{N}_f"] = g
    # vector reductions and updates (include/vecops.hpp)
    M = 101
    A, B, C = (rng.uniform(-1, 1, 2 * M) for _ in range(3))
    Wv = rng.uniform(0, 2, M)
    out["vec_A"], out["vec_B"], out["vec_C"], out["vec_W"] = A, B, C, Wv
    out["vec_doudot"] = R.ref_vec_doudot(M, P(A), P(Wv))
    out["vec_tridot_nn"] = R.ref_vec_tridot_nn(M, P(A), P(B), P(Wv))
    out["vec_shift_window"] = R.ref_vec_shift_window(M, P(A), P(B), P(C), P(Wv))
    out["vec_shift_diff_origin"] = R.ref_vec_shift_diff_origin(M, P(A), P(B), P(Wv))
    for add in (0, 1):
        for cj in (0, 1):
            a = A.copy()
            R.ref_vec_addsub(M, P(a), P(B), add, cj)
            out[f"vec_addsub_{add}{cj}"] = a
            a = A.copy()
            R.ref_vec_muladdsub(M, P(a), P(B), P(C), add, cj)
            out[f"vec_muladdsub_{add}{cj}"] = a
    # wrap and image helpers (include/utils.hpp:58-105)
    L = 10.0
    mm_x = np.array([-25.0, -10.0, -1e-17, -0.3, 0.0, 3.3, 9.999999999999998, 10.0, 10.5, 31.0])
    out["my_mod_L"] = L
    out["my_mod_x"] = mm_x
    out["my_mod"] = np.array([R.ref_my_mod(v, L) for v in mm_x])
    ps_cases = np.array([[1.25, 8.75, 2.5, 2.5], [8.75, 1.25, 2.5, 2.5], [3.75, 6.25, 2.5, 2.5],
                         [0.625, 7.5, 1.25, 5.0], [9.375, 2.5, 1.25, 5.0], [5.0, 5.0, 2.5, 2.5]])
    out["periodic_shift_cases"] = ps_cases
    out["periodic_shift"] = np.array([R.ref_periodic_shift(a, b, L, c, d) for a, b, c, d in ps_cases])
    # random_init stream (include/utils.hpp:122-129)
    ri = np.zeros(64)
    R.ref_random_init(64, 0.0, 20.0, P(ri))
    out["random_init_0_20"] = ri
    np.savez_compressed(os.path.join(HERE, "reference_math.npz"), **out)

    # Ewald known answer (test/ewald_test.cpp:11-157), read as text
    src = open(os.path.join(REF, "test", "ewald_test.cpp")).read()
    qtxt = re.search(r"double q_array\[\] = \{([^}]*)\}", src).group(1)
    q = [float(v) for v in qtxt.split(",") if v.strip()]
    rtxt = re.search(r"double r_array\[\]\[3\] = \{(.*?)\};", src, re.S).group(1)
    r = [[float(v) for v in m.split(",")] for m in re.findall(r"\{([^{}]*)\}", rtxt)]
    val = float(re.search(r"EXPECT_NEAR\(E / \(4 \* M_PI\), (-?[0-9.eE+-]+), 1e-10\)", src).group(1))
    alphas = [float(v) for v in re.search(r"alphas = \{([^}]*)\}", src).group(1).split(",")]
    with open(os.path.join(HERE, "ewald_known_answer.json"), "w") as fh:
        json.dump({"source": "test/ewald_test.cpp:11-157", "L": 100.0, "s": 5.0, "alphas": alphas,
                   "E_over_4pi": val, "tolerance": 1e-10, "q": q, "r": r, "potential_point": [10.0, 10.0, 10.0]},
                  fh, indent=0)
    print("wrote", len(out), "arrays;", len(q), "charges")


if __name__ == "__main__":
    sys.exit(main())
