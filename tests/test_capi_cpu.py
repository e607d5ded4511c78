"""CPU checks of the product boundary: the CUDA library loads, exports every
entry point include/hpdmk.h declares, validates its inputs the way the
reference does (errors instead of exceptions), and its host-side PSWF
set-up matches the reference's golden vectors. No compute call needs a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import pdmk4mc_b200 as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(ROOT, "tests", "golden", "reference_math.npz"))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "hpdmk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(hpdmk_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = P.load_library()
    names = _declared_functions()
    assert "hpdmk_tree_create" in names and "hpdmk_eval_shift_energy" in names
    for n in names:
        assert hasattr(lib, n), n


def test_params_struct_layout_matches_reference():
    # int, int, double, double, enum(int) -> 32 bytes, as the reference's struct
    assert ctypes.sizeof(P.tree._Params) == 32
    assert P.tree._Params.L.offset == 8 and P.tree._Params.init.offset == 24
    d = P.HPDMKParams()
    assert (d.n_per_leaf, d.digits, d.prolate_order, d.init) == (200, 3, 16, P.PROXY)


@pytest.mark.parametrize("kw,code", [
    (dict(digits=5), 1),                      # unsupported digits (src/tree.cpp:25-28)
    (dict(digits=9, init=P.PROXY), 1),        # PROXY above 3 digits (src/upward_pass.cpp:9-14)
    (dict(L=-1.0), 1),
    (dict(n_per_leaf=0), 1),
])
def test_bad_params_rejected(kw, code):
    base = dict(n_per_leaf=10, digits=6, L=10.0, init=P.DIRECT)
    base.update(kw)
    r = np.full(30, 1.0)
    q = np.ones(10)
    with pytest.raises(P.HPDMKError) as e:
        P.HPDMKPtTree(P.HPDMKParams(**base), r, q)
    assert e.value.code == code


@pytest.mark.parametrize("bad", ["outside", "negative", "nan_q"])
def test_bad_inputs_rejected(bad):
    r = np.full(30, 1.0)
    q = np.ones(10)
    if bad == "outside":
        r[4] = 10.0
    elif bad == "negative":
        r[7] = -1e-9
    else:
        q[3] = np.nan
    with pytest.raises(P.HPDMKError) as e:
        P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=10, digits=6, L=10.0, init=P.DIRECT), r, q)
    assert e.value.code == 2


def test_reference_c_entry_point_is_safe_on_bad_input():
    lib = P.load_library()
    cp = P.tree._Params(10, 7, 10.0, 16.0, P.DIRECT)
    r = np.full(30, 1.0)
    q = np.ones(10)
    lib.hpdmk_tree_create(0, cp, 10, r.ctypes.data_as(P.tree._dp), q.ctypes.data_as(P.tree._dp))
    assert lib.hpdmk_last_error() == 1


@pytest.mark.parametrize("digits", [3, 6, 9, 12])
def test_host_prolate_setup_matches_reference(digits):
    xs = G[f"d{digits}_psi0_x"]
    out, psi = P.prolate_setup(digits, xs)
    c, lam, c0r, diff0, nw, nd = out
    assert c == G[f"d{digits}_c"]
    assert int(nd) == int(G[f"d{digits}_n_diff"])
    assert int(nw) == int(np.floor(2 * c / np.pi))
    assert abs(lam / G[f"d{digits}_lambda"] - 1) < 1e-12
    p0 = G[f"d{digits}_psi0"][0]
    assert abs(c0r - G[f"d{digits}_C0"] / p0) < 1e-13
    assert abs(diff0 / G[f"d{digits}_diff0"] - 1) < 1e-12
    np.testing.assert_allclose(psi, G[f"d{digits}_psi0"] / p0, rtol=0, atol=1e-14)


def test_read_particle_info(tmp_path):
    # the reference's read_particle_info (src/utils.cpp:14-28): the first line
    # is a header; a line counts when it starts with four numbers x y z q
    f = tmp_path / "system.xyzq"
    f.write_text("x y z q\n1.5 2 3 1\nnot a particle\n4 5 6 -1 trailing words\n\n7 8\n0.25 0.5 0.75 2e-1\n")
    r, q = P.read_particle_info(str(f))
    np.testing.assert_array_equal(r, [1.5, 2, 3, 4, 5, 6, 0.25, 0.5, 0.75])
    np.testing.assert_array_equal(q, [1, -1, 0.2])
    g = tmp_path / "header_only.xyzq"
    g.write_text("x y z q\n")
    r, q = P.read_particle_info(str(g))
    assert r.size == 0 and q.size == 0
    with pytest.raises(P.HPDMKError) as e:
        P.read_particle_info(str(tmp_path / "missing.xyzq"))
    assert e.value.code == 2


def test_tuning_table_lookup(tmp_path):
    # the autotuner's JSON table: the same size bucket (floor(log2 N)) wins,
    # else the nearest bucket of the same digits and precision, else defaults
    f = tmp_path / "tuning.json"
    f.write_text('[\n  {"digits": 9, "precision": 1, "n_log2": 16, "ksplit": 2048, "ksplit_root": 1024, '
                 '"inc_waves": 8, "res_ny_max": 4},\n'
                 '  {"digits": 9, "precision": 1, "n_log2": 19, "ksplit": 8192, "ksplit_root": 4096, '
                 '"inc_waves": 2, "res_ny_max": 2},\n'
                 '  {"digits": 9, "precision": 0, "n_log2": 19, "ksplit": 16384}\n]\n')
    lib = P.load_library()
    out = np.zeros(4, np.int32)

    def look(d, p, n):
        assert lib.hpdmk_debug_tuning_lookup(str(f).encode(), d, p, n, out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_int))) == 0
        return out.tolist()
    assert look(9, 1, 100000) == [2048, 1024, 8, 4]      # 2^16 <= 1e5 < 2^17
    assert look(9, 1, 1000000) == [8192, 4096, 2, 2]     # 2^19 <= 1e6 < 2^20
    assert look(9, 1, 4000000) == [8192, 4096, 2, 2]     # nearest bucket
    assert look(9, 0, 1000000) == [16384, 2048, 4, 8]    # missing fields keep their defaults
    assert look(6, 1, 1000000) == [4096, 2048, 4, 8]     # no entry: defaults
    (tmp_path / "bad.json").write_text("not json at all {")
    assert lib.hpdmk_debug_tuning_lookup(str(tmp_path / "bad.json").encode(), 9, 1, 1000, out.ctypes.data_as(
        ctypes.POINTER(ctypes.c_int))) == 0 and out.tolist() == [4096, 2048, 4, 8]
