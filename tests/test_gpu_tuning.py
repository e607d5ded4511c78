"""The autotuner (hpdmk_autotune, no reference counterpart): tuning changes
only how the work is split, so the energies before and after agree to
rounding, the table it writes holds the tree's entry, and hand-set values
are clamped to the supported ranges."""
import json

import numpy as np
import pytest

import pdmk4mc_b200 as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [P.PRECISION_FP64, P.PRECISION_MIXED])
def test_autotune_keeps_energies(tmp_path, precision):
    n, L = 20000, 27.1
    rng = np.random.default_rng(4)
    r = rng.uniform(0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    t = P.HPDMKPtTree(P.HPDMKParams(n_per_leaf=50, digits=9, L=L, init=P.DIRECT), r, q, precision=precision)
    try:
        t.form_outgoing_pw()
        t.form_incoming_pw()
        e0 = t.eval_energy_parts()
        path = tmp_path / "tuning.json"
        chosen, times = t.autotune(str(path), reps=2)
        assert t.tuning() == chosen and all(v > 0 for v in times.values())
        e1 = t.eval_energy_parts()
        assert np.all(np.abs(e1 - e0) <= 1e-11 * abs(e0.sum())), (e0, e1)
        table = json.loads(path.read_text())
        entry = [x for x in table if x["digits"] == 9 and x["precision"] == precision and x["n_log2"] == 14]
        assert len(entry) == 1 and {k: entry[0][k] for k in chosen} == chosen
        # hand-set values are clamped; the energy stays put
        t.set_tuning(ksplit=10, res_ny_max=100)
        assert t.tuning()["ksplit"] == 256 and t.tuning()["res_ny_max"] == 8
        t.form_outgoing_pw()
        t.form_incoming_pw()
        e2 = t.eval_energy_parts()
        assert np.all(np.abs(e2 - e0) <= 1e-11 * abs(e0.sum())), (e0, e2)
    finally:
        t.close()
