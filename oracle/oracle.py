"""ORACLE — test infrastructure only.

ctypes front end of oracle/liboracle.so (the CPU restatement of the
reference's DMK energy path, oracle_core.cpp) with the set-up constants from
oracle/pswf.py. Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may import this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import pswf

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_long)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_uint64)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_long, _dp, _dp, ctypes.c_int, _dp,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp,
                                ctypes.c_int, ctypes.c_int]
        L.or_destroy.argtypes = [ctypes.c_void_p]
        L.or_info.argtypes = [ctypes.c_void_p, _lp]
        L.or_form_outgoing.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.or_form_incoming.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.or_energy.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.or_energy_direct.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.or_shift.restype = ctypes.c_double
        L.or_shift.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
        L.or_update.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_int]
        L.or_tree_nodes.argtypes = [ctypes.c_void_p, _ip, _up, _ip, _lp]
        L.or_tree_neighbors.argtypes = [ctypes.c_void_p, _ip, _ip]
        L.or_sorted_order.argtypes = [ctypes.c_void_p, _lp]
        L.or_positions.argtypes = [ctypes.c_void_p, _dp]
        L.or_get_pw.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, _dp]
        L.or_get_W.argtypes = [ctypes.c_void_p, _dp]
        L.or_get_D.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.or_leaf_path.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, _lp, _ip]
        L.or_ewald_energy.restype = ctypes.c_double
        L.or_ewald_energy.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_long, _dp, _dp,
                                      ctypes.c_int]
        L.or_ewald_potential.restype = ctypes.c_double
        L.or_ewald_potential.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_long, _dp, _dp,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_long, ctypes.c_int]
        L.or_random_init.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_double, _dp]
        L.or_reference_trials.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_long, _dp, _lp]
        L.or_ewald_create.restype = ctypes.c_void_p
        L.or_ewald_create.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_long, _dp, _dp,
                                      ctypes.c_int]
        L.or_ewald_destroy.argtypes = [ctypes.c_void_p]
        L.or_ewald_move.restype = ctypes.c_double
        L.or_ewald_move.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int]
        L.or_nudft_halfplane.argtypes = [ctypes.c_long, _dp, _dp, _dp, _dp, ctypes.c_int, _dp]
        L.or_nudft_single.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int, _dp]
        L.or_shift_phases.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _dp]
        L.or_res_kernel.restype = ctypes.c_double
        L.or_res_kernel.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double]
        L.or_my_mod.restype = ctypes.c_double
        L.or_my_mod.argtypes = [ctypes.c_double, ctypes.c_double]
        L.or_periodic_shift.restype = ctypes.c_int
        L.or_periodic_shift.argtypes = [ctypes.c_double] * 5
        _LIB = L
    return _LIB


def random_init(n: int, lo: float, hi: float) -> np.ndarray:
    """The reference's random_init stream (default-seeded std::mt19937)."""
    out = np.empty(n, dtype=np.float64)
    lib().or_random_init(n, lo, hi, _p(out))
    return out


def reference_trials(ntrials: int, L: float, n: int):
    """(displacements [ntrials,3], particle indices) of the reference tests' move stream."""
    d = np.zeros(3 * ntrials)
    idx = np.zeros(ntrials, np.int64)
    lib().or_reference_trials(ntrials, L, n, _p(d), _p(idx, _lp))
    return d.reshape(ntrials, 3), idx


def reference_test_system(n: int, L: float):
    """Positions and neutralised charges exactly as the reference's tests make them
    (random_init(r,0,L); random_init(q,-1,1); unify_charge), test/hpdmk_test.cpp:24-33."""
    r = random_init(3 * n, 0.0, L)
    q = random_init(n, -1.0, 1.0)
    q = q - q.sum() / n
    return r, q


def ewald_energy(L, r, q, s=5.0, alpha=1.0, nthreads=None):
    r = np.ascontiguousarray(r, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().or_ewald_energy(L, s, alpha, len(q), _p(r), _p(q), nthreads or os.cpu_count())


def ewald_potential(L, r, q, i, x, s=5.0, alpha=1.0, nthreads=None):
    """Ewald potential at point x of all particles except i (src/ewald.cpp:281-308,
    compute_potential, with particle i left out)."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    return lib().or_ewald_potential(L, s, alpha, len(q), _p(r), _p(q), x[0], x[1], x[2], int(i),
                                    nthreads or os.cpu_count())


def ewald_shift(L, r, q, i, d, s=5.0, alpha=1.0, nthreads=None):
    """Exact Ewald energy change of moving particle i by d (wrapped into the box):
    q_i [phi_{-i}(new) - phi_{-i}(old)]."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    nt = nthreads or os.cpu_count()
    old = r[3 * i:3 * i + 3].copy()
    new = np.mod(old + np.asarray(d, dtype=np.float64), L)
    po = lib().or_ewald_potential(L, s, alpha, len(q), _p(r), _p(q), old[0], old[1], old[2], i, nt)
    pn = lib().or_ewald_potential(L, s, alpha, len(q), _p(r), _p(q), new[0], new[1], new[2], i, nt)
    return q[i] * (pn - po)


class EwaldMC:
    """FP64 Ewald state for sequential moves: exact energy change per move in O(N + K)."""

    def __init__(self, L, r, q, s=5.0, alpha=1.0, nthreads=None):
        r = np.ascontiguousarray(r, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        self.h = lib().or_ewald_create(L, s, alpha, len(q), _p(r), _p(q), nthreads or os.cpu_count())

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_ewald_destroy(self.h)
            self.h = None

    def shift(self, i, d):
        return lib().or_ewald_move(self.h, int(i), float(d[0]), float(d[1]), float(d[2]), 0)

    def move(self, i, d):
        return lib().or_ewald_move(self.h, int(i), float(d[0]), float(d[1]), float(d[2]), 1)


class OracleTree:
    """Mirror of the reference's HPDMKPtTree<double> (include/tree.hpp:29-132) on the CPU."""

    def __init__(self, L, n_per_leaf, digits, r, q, nthreads=None):
        self.k = pswf.constants(digits)
        self.L = float(L)
        self.nthreads = nthreads or os.cpu_count()
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        leg = np.ascontiguousarray(self.k["legendre"], dtype=np.float64)
        poly = np.ascontiguousarray(self.k["poly_horner"], dtype=np.float64)
        self.h = lib().or_create(self.L, int(n_per_leaf), int(digits), len(q), _p(r), _p(q), len(leg), _p(leg),
                                 self.k["c"], self.k["lam"], self.k["C0"], self.k["diff0"], len(poly), _p(poly),
                                 self.k["n_window"], self.k["n_diff"])
        info = np.zeros(7, dtype=np.int64)
        lib().or_info(self.h, _p(info, _lp))
        self.max_depth, self.n_nodes, self.n, self.dims_window, self.dims_diff, self.n_window, self.n_diff = map(int, info)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def form_outgoing_pw(self):
        lib().or_form_outgoing(self.h, self.nthreads)

    def form_incoming_pw(self):
        lib().or_form_incoming(self.h, self.nthreads)

    def eval_energy_parts(self):
        p = np.zeros(3)
        lib().or_energy(self.h, self.nthreads, _p(p))
        return p

    def eval_energy(self):
        return float(self.eval_energy_parts().sum())

    def eval_energy_direct_parts(self):
        p = np.zeros(3)
        lib().or_energy_direct(self.h, self.nthreads, _p(p))
        return p

    def eval_shift_energy(self, i, dx, dy, dz, parts=False):
        p = np.zeros(5)
        v = lib().or_shift(self.h, int(i), float(dx), float(dy), float(dz), _p(p))
        return (v, p) if parts else v

    def update_shift(self, i, dx, dy, dz):
        lib().or_update(self.h, int(i), float(dx), float(dy), float(dz), 1)

    def tree_nodes(self):
        lv = np.zeros(self.n_nodes, np.int32)
        pf = np.zeros(self.n_nodes, np.uint64)
        lf = np.zeros(self.n_nodes, np.int32)
        ct = np.zeros(self.n_nodes, np.int64)
        lib().or_tree_nodes(self.h, _p(lv, _ip), _p(pf, _up), _p(lf, _ip), _p(ct, _lp))
        return lv, pf, lf, ct

    def tree_neighbors(self):
        col = np.zeros((self.n_nodes, 27), np.int32)
        cg = np.zeros((self.n_nodes, 8), np.int32)
        lib().or_tree_neighbors(self.h, _p(col, _ip), _p(cg, _ip))
        return col, cg

    def sorted_order(self):
        o = np.zeros(self.n, np.int64)
        lib().or_sorted_order(self.h, _p(o, _lp))
        return o

    def positions(self):
        r = np.zeros(3 * self.n)
        lib().or_positions(self.h, _p(r))
        return r

    def pw(self, node, which="out"):
        dims = self.dims_window if node == 0 else self.dims_diff
        o = np.zeros(2 * dims)
        lib().or_get_pw(self.h, int(node), 0 if which == "out" else 1, _p(o))
        return o[0::2] + 1j * o[1::2]

    def window_matrix(self):
        o = np.zeros(self.dims_window)
        lib().or_get_W(self.h, _p(o))
        return o

    def difference_matrix(self, level):
        o = np.zeros(self.dims_diff)
        lib().or_get_D(self.h, int(level), _p(o))
        return o

    def leaf_path(self, x, y, z):
        p = np.zeros(32, np.int64)
        d = ctypes.c_int()
        lib().or_leaf_path(self.h, x, y, z, _p(p, _lp), ctypes.byref(d))
        return p[:d.value]
