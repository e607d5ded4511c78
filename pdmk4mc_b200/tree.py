"""Python mirror of the reference's HPDMKPtTree<double> (include/tree.hpp:29-132)
over the C-ABI of libhpdmk_b200.so (include/hpdmk.h).

    params = HPDMKParams(n_per_leaf=10, digits=9, L=20.0, init=DIRECT)
    tree = HPDMKPtTree(params, r_src, charge)    # r_src: [3n] xyz-interleaved in [0, L)
    tree.form_outgoing_pw(); tree.form_incoming_pw()
    E = tree.eval_energy()
    dE = tree.eval_shift_energy(i, dx, dy, dz)
    tree.update_shift(i, dx, dy, dz)

Errors of the library (the reference's exceptions) raise HPDMKError.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

DIRECT = 1
PROXY = 2
STATIC_MAX_MOVES = 4096  # HPDMK_STATIC_MAX_MOVES in include/hpdmk.h
MC_PERSISTENT = 0  # HPDMK_MC_PERSISTENT
MC_GRAPH = 1  # HPDMK_MC_GRAPH
PRECISION_FP64 = 0  # HPDMK_PRECISION_FP64
PRECISION_MIXED = 1  # HPDMK_PRECISION_MIXED: outgoing expansions on the tensor cores from int8 slices

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_long)
_ip = ctypes.POINTER(ctypes.c_int)
_ullp = ctypes.POINTER(ctypes.c_ulonglong)


class HPDMKError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"hpdmk error {code}: {message}")
        self.code = code


class _Params(ctypes.Structure):
    # include/hpdmk.h: struct HPDMKParams (same layout as the reference's)
    _fields_ = [("n_per_leaf", ctypes.c_int), ("digits", ctypes.c_int), ("L", ctypes.c_double),
                ("prolate_order", ctypes.c_double), ("init", ctypes.c_int)]


class _ExtParams(ctypes.Structure):
    _fields_ = [("leaf_slack", ctypes.c_int), ("pool_capacity", ctypes.c_int), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("stream", ctypes.c_void_p)]


@dataclass
class HPDMKParams:
    """include/hpdmk.h:11-17 of the reference, with its defaults."""
    n_per_leaf: int = 200
    digits: int = 3
    L: float = 1.0
    prolate_order: float = 16
    init: int = PROXY


def library_path() -> str:
    return os.environ.get("PDMK_B200_LIB", os.path.join(_HERE, "libhpdmk_b200.so"))


def launch_count() -> int:
    """Kernels this library has launched since it was loaded (graph-run ones included)."""
    v = ctypes.c_longlong(0)
    _check(load_library().hpdmk_get_launch_count(ctypes.byref(v)))
    return int(v.value)


def replicas_mc_run(trees, idx, disp, u, beta):
    """Metropolis sequences of many trees in one launch (one block per tree).
    idx, u: [n_trees, m]; disp: [n_trees, m, 3]. Returns (dE, accepted), [n_trees, m]."""
    nt = len(trees)
    idx = np.ascontiguousarray(idx, dtype=np.int64).reshape(nt, -1)
    m = idx.shape[1]
    disp = np.ascontiguousarray(disp, dtype=np.float64).reshape(nt * m * 3)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(nt * m)
    hs = (ctypes.c_void_p * nt)(*[t._h for t in trees])
    dE = np.zeros(nt * m)
    acc = np.zeros(nt * m, np.int32)
    _check(load_library().hpdmk_replicas_mc_run(nt, hs, m, _p(idx, _lp), _p(disp), _p(u), float(beta), _p(dE),
                                                _p(acc, _ip)))
    return dE.reshape(nt, m), acc.reshape(nt, m)


def replicas_energy(trees):
    """Full energy (outgoing, incoming, energy) of each tree, several in flight at once."""
    nt = len(trees)
    hs = (ctypes.c_void_p * nt)(*[t._h for t in trees])
    e = np.zeros(nt)
    _check(load_library().hpdmk_replicas_energy(nt, hs, _p(e)))
    return e


def read_particle_info(path):
    """The reference's read_particle_info (src/utils.cpp:14-28): a header line,
    then "x y z q" per line. Returns (r[3n] xyz-interleaved, q[n])."""
    L = load_library()
    n = ctypes.c_long(0)
    p = os.fsencode(path)
    _check(L.hpdmk_read_particle_info(p, ctypes.byref(n), None, None, 0))
    r = np.zeros(3 * n.value)
    q = np.zeros(n.value)
    _check(L.hpdmk_read_particle_info(p, ctypes.byref(n), _p(r), _p(q), n.value))
    return r, q


def load_library():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"libhpdmk_b200.so not built: {path} (run __graft_entry__.build() or make -C "
                          f"pdmk4mc_b200/csrc)")
    L = ctypes.CDLL(path)
    L.hpdmk_tree_create.restype = None
    L.hpdmk_tree_create.argtypes = [ctypes.c_int, _Params, ctypes.c_int, _dp, _dp]
    L.hpdmk_tree_init.restype = ctypes.c_void_p
    L.hpdmk_tree_init.argtypes = [ctypes.c_int, _Params, ctypes.c_int, _dp, _dp]
    L.hpdmk_tree_init_ext.restype = ctypes.c_void_p
    L.hpdmk_tree_init_ext.argtypes = [ctypes.c_int, _Params, ctypes.POINTER(_ExtParams), ctypes.c_int, _dp, _dp]
    L.hpdmk_tree_init_device.restype = ctypes.c_void_p
    L.hpdmk_tree_init_device.argtypes = [ctypes.c_int, _Params, ctypes.POINTER(_ExtParams), ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]
    L.hpdmk_get_stream.restype = ctypes.c_int
    L.hpdmk_get_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.hpdmk_replicas_mc_run.restype = ctypes.c_int
    L.hpdmk_replicas_mc_run.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, _lp, _dp, _dp,
                                        ctypes.c_double, _dp, _ip]
    L.hpdmk_eval_potential.restype = ctypes.c_int
    L.hpdmk_eval_potential.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _dp, _dp]
    L.hpdmk_replicas_energy.restype = ctypes.c_int
    L.hpdmk_replicas_energy.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), _dp]
    L.hpdmk_tree_rebuild.restype = ctypes.c_int
    L.hpdmk_tree_rebuild.argtypes = [ctypes.c_void_p]
    L.hpdmk_set_rebuild_policy.restype = ctypes.c_int
    L.hpdmk_set_rebuild_policy.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.hpdmk_tree_drift.restype = ctypes.c_int
    L.hpdmk_tree_drift.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int)]
    L.hpdmk_ewald_energy.restype = ctypes.c_int
    L.hpdmk_ewald_energy.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.hpdmk_set_mc_mode.restype = ctypes.c_int
    L.hpdmk_set_mc_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.hpdmk_set_timing.restype = ctypes.c_int
    L.hpdmk_set_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.hpdmk_get_timing.restype = ctypes.c_int
    L.hpdmk_get_timing.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int]
    L.hpdmk_get_launch_count.restype = ctypes.c_int
    L.hpdmk_get_launch_count.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    L.hpdmk_get_update_bytes.restype = ctypes.c_int
    L.hpdmk_get_update_bytes.argtypes = [ctypes.c_void_p, _dp]
    L.hpdmk_tree_destroy.restype = None
    L.hpdmk_tree_destroy.argtypes = [ctypes.c_void_p]
    for name in ("hpdmk_form_outgoing_pw", "hpdmk_form_incoming_pw", "hpdmk_synchronize"):
        getattr(L, name).restype = ctypes.c_int
        getattr(L, name).argtypes = [ctypes.c_void_p]
    L.hpdmk_eval_energy.restype = ctypes.c_int
    L.hpdmk_eval_energy.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
    L.hpdmk_energy.restype = ctypes.c_int
    L.hpdmk_energy.argtypes = [ctypes.c_void_p, _dp]
    L.hpdmk_eval_shift_energy.restype = ctypes.c_int
    L.hpdmk_eval_shift_energy.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, _dp]
    L.hpdmk_debug_shift_parts.restype = ctypes.c_int
    L.hpdmk_debug_shift_parts.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, _dp]
    L.hpdmk_update_shift.restype = ctypes.c_int
    L.hpdmk_update_shift.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double]
    L.hpdmk_eval_shift_energy_batch.restype = ctypes.c_int
    L.hpdmk_eval_shift_energy_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _dp, _dp]
    L.hpdmk_eval_shift_energy_batch_static.restype = ctypes.c_int
    L.hpdmk_eval_shift_energy_batch_static.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _dp, _dp]
    L.hpdmk_eval_shift_energy_batch_device.restype = ctypes.c_int
    L.hpdmk_eval_shift_energy_batch_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]
    L.hpdmk_mc_run.restype = ctypes.c_int
    L.hpdmk_mc_run.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _dp, _dp, ctypes.c_double, _dp, _ip]
    L.hpdmk_mc_run_device.restype = ctypes.c_int
    L.hpdmk_mc_run_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.hpdmk_get_positions.restype = ctypes.c_int
    L.hpdmk_get_positions.argtypes = [ctypes.c_void_p, _dp]
    L.hpdmk_tree_info.restype = ctypes.c_int
    L.hpdmk_tree_info.argtypes = [ctypes.c_void_p, _lp]
    L.hpdmk_read_particle_info.restype = ctypes.c_int
    L.hpdmk_read_particle_info.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_long), _dp, _dp, ctypes.c_long]
    L.hpdmk_autotune.restype = ctypes.c_int
    L.hpdmk_autotune.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, _ip, _dp]
    L.hpdmk_get_tuning.restype = ctypes.c_int
    L.hpdmk_get_tuning.argtypes = [ctypes.c_void_p, _ip]
    L.hpdmk_set_tuning.restype = ctypes.c_int
    L.hpdmk_set_tuning.argtypes = [ctypes.c_void_p, _ip]
    L.hpdmk_debug_tuning_lookup.restype = ctypes.c_int
    L.hpdmk_debug_tuning_lookup.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_long, _ip]
    L.hpdmk_last_error.restype = ctypes.c_int
    L.hpdmk_last_error.argtypes = []
    L.hpdmk_last_error_message.restype = ctypes.c_char_p
    L.hpdmk_last_error_message.argtypes = []
    L.hpdmk_debug_nodes.restype = ctypes.c_int
    L.hpdmk_debug_nodes.argtypes = [ctypes.c_void_p, _ip, _ullp, _ip, _lp]
    L.hpdmk_debug_neighbors.restype = ctypes.c_int
    L.hpdmk_debug_neighbors.argtypes = [ctypes.c_void_p, _ip, _ip]
    L.hpdmk_debug_sorted_order.restype = ctypes.c_int
    L.hpdmk_debug_sorted_order.argtypes = [ctypes.c_void_p, _lp]
    L.hpdmk_debug_pw.restype = ctypes.c_int
    L.hpdmk_debug_pw.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, _dp]
    L.hpdmk_debug_kernels.restype = ctypes.c_int
    L.hpdmk_debug_kernels.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    L.hpdmk_debug_prolate.restype = ctypes.c_int
    L.hpdmk_debug_prolate.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp]
    _LIB = L
    return L


def prolate_setup(digits: int, x=None):
    """Host-side PSWF set-up of the library: (c, lambda, C0/psi0(0), diff0, n_window, n_diff), psi0(x)/psi0(0)."""
    L = load_library()
    out = np.zeros(6)
    x = np.ascontiguousarray(np.zeros(0) if x is None else x, dtype=np.float64)
    psi = np.zeros_like(x)
    _check(L.hpdmk_debug_prolate(int(digits), _p(out), int(x.size), _p(x), _p(psi)))
    return out, psi


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _check(rc):
    if rc != 0:
        L = load_library()
        raise HPDMKError(rc, L.hpdmk_last_error_message().decode(errors="replace"))


class HPDMKPtTree:
    """Device-resident DMK tree (reference: HPDMKPtTree<double>, include/tree.hpp:29-132)."""

    def __init__(self, params: HPDMKParams, r_src, charge, leaf_slack: int = 8, pool_capacity: int = 4096,
                 device: int = 0, stream=None, device_inputs=None, precision: int = PRECISION_FP64):
        """r_src / charge: host arrays; or, with device_inputs=(d_r_ptr, d_q_ptr, n), device pointers.
        precision: PRECISION_FP64 (default) or PRECISION_MIXED."""
        L = load_library()
        self.params = params
        cp = _Params(int(params.n_per_leaf), int(params.digits), float(params.L), float(params.prolate_order),
                     int(params.init))
        ext = _ExtParams(int(leaf_slack), int(pool_capacity), int(precision), int(device), stream)
        if device_inputs is not None:
            d_r, d_q, n = device_inputs
            self._h = L.hpdmk_tree_init_device(0, cp, ctypes.byref(ext), int(n), d_r, d_q)
        else:
            r = np.ascontiguousarray(r_src, dtype=np.float64).reshape(-1)
            q = np.ascontiguousarray(charge, dtype=np.float64).reshape(-1)
            if r.size != 3 * q.size:
                raise ValueError("r_src must hold 3 coordinates per charge")
            n = q.size
            self._h = L.hpdmk_tree_init_ext(0, cp, ctypes.byref(ext), int(n), _p(r), _p(q))
        if not self._h:
            _check(L.hpdmk_last_error())
        self.n = int(n)
        self.L = float(params.L)
        self._refresh_info()

    def _refresh_info(self):
        info = np.zeros(5, np.int64)
        _check(load_library().hpdmk_tree_info(self._h, _p(info, _lp)))
        self.max_depth, self.n_nodes, _, self.dims_window, self.dims_diff = (int(v) for v in info)

    def close(self):
        if getattr(self, "_h", None):
            load_library().hpdmk_tree_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    def form_outgoing_pw(self):
        _check(load_library().hpdmk_form_outgoing_pw(self._h))
        if getattr(self, "_rebuild_factor", 0.0) > 0.0:
            self._refresh_info()  # the rebuild policy may have re-binned the tree

    def set_rebuild_policy(self, leaf_factor):
        """With leaf_factor > 1, every form_outgoing_pw first rebuilds the tree
        when a leaf holds more than leaf_factor * n_per_leaf particles or a
        refined node below level 2 fewer than n_per_leaf / leaf_factor; 0 turns
        the check off (hpdmk_set_rebuild_policy)."""
        _check(load_library().hpdmk_set_rebuild_policy(self._h, float(leaf_factor)))
        self._rebuild_factor = float(leaf_factor)

    def drift(self):
        """(largest leaf count, smallest refined-node count below level 2,
        rebuilds made by the policy)."""
        a, b, c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(load_library().hpdmk_tree_drift(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def form_incoming_pw(self):
        _check(load_library().hpdmk_form_incoming_pw(self._h))

    def eval_energy_parts(self):
        e, w, d, r = (ctypes.c_double() for _ in range(4))
        _check(load_library().hpdmk_eval_energy(self._h, ctypes.byref(e), ctypes.byref(w), ctypes.byref(d),
                                                ctypes.byref(r)))
        return np.array([w.value, d.value, r.value])

    def eval_energy(self) -> float:
        return float(self.eval_energy_parts().sum())

    def eval_energy_window(self):
        return float(self.eval_energy_parts()[0])

    def eval_energy_diff(self):
        return float(self.eval_energy_parts()[1])

    def eval_energy_res(self):
        return float(self.eval_energy_parts()[2])

    def eval_shift_energy(self, i, dx, dy, dz) -> float:
        out = ctypes.c_double()
        _check(load_library().hpdmk_eval_shift_energy(self._h, int(i), float(dx), float(dy), float(dz),
                                                      ctypes.byref(out)))
        return out.value

    def eval_shift_energy_parts(self, i, dx, dy, dz):
        """(window, difference, residual at target, residual at origin, self term)."""
        p = np.zeros(5)
        _check(load_library().hpdmk_debug_shift_parts(self._h, int(i), float(dx), float(dy), float(dz), _p(p)))
        return p

    def update_shift(self, i, dx, dy, dz):
        _check(load_library().hpdmk_update_shift(self._h, int(i), float(dx), float(dy), float(dz)))

    def eval_shift_energy_batch(self, idx, disp):
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        disp = np.ascontiguousarray(disp, dtype=np.float64).reshape(-1)
        out = np.zeros(idx.size)
        _check(load_library().hpdmk_eval_shift_energy_batch(self._h, int(idx.size), _p(idx, _lp), _p(disp),
                                                            _p(out)))
        return out

    def eval_shift_energy_batch_static(self, idx, disp):
        """eval_shift_energy_batch through the fixed static device buffer:
        no device allocation in the call, at most STATIC_MAX_MOVES candidates."""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        disp = np.ascontiguousarray(disp, dtype=np.float64).reshape(-1)
        out = np.zeros(idx.size)
        _check(load_library().hpdmk_eval_shift_energy_batch_static(self._h, int(idx.size), _p(idx, _lp), _p(disp),
                                                                   _p(out)))
        return out

    def mc_run(self, idx, disp, u, beta):
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        disp = np.ascontiguousarray(disp, dtype=np.float64).reshape(-1)
        u = np.ascontiguousarray(u, dtype=np.float64)
        dE = np.zeros(idx.size)
        acc = np.zeros(idx.size, np.int32)
        _check(load_library().hpdmk_mc_run(self._h, int(idx.size), _p(idx, _lp), _p(disp), _p(u), float(beta),
                                           _p(dE), _p(acc, _ip)))
        return dE, acc

    def mc_run_device(self, n, d_idx_ptr, d_disp_ptr, d_u_ptr, beta, d_dE_ptr, d_acc_ptr):
        _check(load_library().hpdmk_mc_run_device(self._h, int(n), d_idx_ptr, d_disp_ptr, d_u_ptr, float(beta),
                                                  d_dE_ptr, d_acc_ptr))

    def eval_shift_energy_batch_device(self, m, d_idx_ptr, d_disp_ptr, d_dE_ptr):
        """Candidate batch on device arrays (int32 indices), enqueued on the tree's stream."""
        _check(load_library().hpdmk_eval_shift_energy_batch_device(self._h, int(m), d_idx_ptr, d_disp_ptr, d_dE_ptr))

    TUNING_FIELDS = ("ksplit", "ksplit_root", "inc_waves", "res_ny_max")

    def autotune(self, path=None, reps=3):
        """Search this tree's run-time splits and tiles and record them in the
        tuning table (path None: tuning.json beside the library). Returns
        (chosen {field: value}, {phase: milliseconds})."""
        chosen = np.zeros(4, np.int32)
        times = np.zeros(3)
        p = os.fsencode(path) if path else None
        _check(load_library().hpdmk_autotune(self._h, p, int(reps), _p(chosen, _ip), _p(times)))
        return (dict(zip(self.TUNING_FIELDS, (int(v) for v in chosen))),
                dict(zip(("outgoing_ms", "incoming_ms", "near_field_ms"), (float(v) for v in times))))

    def tuning(self):
        v = np.zeros(4, np.int32)
        _check(load_library().hpdmk_get_tuning(self._h, _p(v, _ip)))
        return dict(zip(self.TUNING_FIELDS, (int(x) for x in v)))

    def set_tuning(self, **kw):
        cur = self.tuning()
        cur.update(kw)
        v = np.array([cur[f] for f in self.TUNING_FIELDS], np.int32)
        _check(load_library().hpdmk_set_tuning(self._h, _p(v, _ip)))

    def synchronize(self):
        _check(load_library().hpdmk_synchronize(self._h))

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        _check(load_library().hpdmk_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def set_timing(self, on: bool):
        _check(load_library().hpdmk_set_timing(self._h, 1 if on else 0))

    def potential(self, idx, field=True):
        """phi = dE/dq at particles idx (E = 1/2 sum q phi) and the field -grad phi."""
        idx = np.ascontiguousarray(idx, dtype=np.int64).reshape(-1)
        phi = np.zeros(idx.size)
        f = np.zeros(3 * idx.size) if field else None
        _check(load_library().hpdmk_eval_potential(self._h, int(idx.size), _p(idx, _lp), _p(phi),
                                                   _p(f) if field else None))
        return (phi, f.reshape(-1, 3)) if field else phi

    def rebuild(self):
        """Re-bin the tree from the current positions and re-form the expansions."""
        _check(load_library().hpdmk_tree_rebuild(self._h))
        self._refresh_info()

    def ewald_energy(self):
        """FP64 Ewald energy of the current particles and its (real, reciprocal, self) parts."""
        e = ctypes.c_double(0.0)
        parts = np.zeros(3)
        _check(load_library().hpdmk_ewald_energy(self._h, ctypes.byref(e), _p(parts)))
        return e.value, parts

    def set_mc_mode(self, mode):
        """MC_PERSISTENT (one cooperative launch, default) or MC_GRAPH (graphs of launch pairs)."""
        _check(load_library().hpdmk_set_mc_mode(self._h, int(mode)))

    def get_timing(self, reset=False):
        """{class: (total ms, launches)} for shift, update, persistent Metropolis and nudft kernels."""
        o = np.zeros(8)
        _check(load_library().hpdmk_get_timing(self._h, _p(o), 1 if reset else 0))
        return {k: (o[2 * c], int(o[2 * c + 1])) for c, k in enumerate(("shift", "update", "mc", "nudft"))}

    def update_work(self):
        """(accepted moves, algorithmic update bytes, dE bytes of the persistent kernel) of the last MC batch."""
        o = np.zeros(3)
        _check(load_library().hpdmk_get_update_bytes(self._h, _p(o)))
        return o

    def positions(self):
        r = np.zeros(3 * self.n)
        _check(load_library().hpdmk_get_positions(self._h, _p(r)))
        return r

    # --- introspection for parity tests
    def tree_nodes(self):
        lv = np.zeros(self.n_nodes, np.int32)
        pf = np.zeros(self.n_nodes, np.uint64)
        lf = np.zeros(self.n_nodes, np.int32)
        ct = np.zeros(self.n_nodes, np.int64)
        _check(load_library().hpdmk_debug_nodes(self._h, _p(lv, _ip), _p(pf, _ullp), _p(lf, _ip), _p(ct, _lp)))
        return lv, pf, lf, ct

    def tree_neighbors(self):
        col = np.zeros((self.n_nodes, 27), np.int32)
        cg = np.zeros((self.n_nodes, 8), np.int32)
        _check(load_library().hpdmk_debug_neighbors(self._h, _p(col, _ip), _p(cg, _ip)))
        return col, cg

    def sorted_order(self):
        o = np.zeros(self.n, np.int64)
        _check(load_library().hpdmk_debug_sorted_order(self._h, _p(o, _lp)))
        return o

    def pw(self, node, which="out"):
        dims = self.dims_window if node == 0 else self.dims_diff
        o = np.zeros(2 * dims)
        _check(load_library().hpdmk_debug_pw(self._h, int(node), 0 if which == "out" else 1, _p(o)))
        return o[0::2] + 1j * o[1::2]

    def window_matrix(self):
        o = np.zeros(self.dims_window)
        _check(load_library().hpdmk_debug_kernels(self._h, 0, _p(o)))
        return o

    def difference_matrix(self, level):
        o = np.zeros(self.dims_diff)
        _check(load_library().hpdmk_debug_kernels(self._h, int(level), _p(o)))
        return o
