"""The demo mechanism sets generated from NMODL files (written for the
tests: tests/golden/mod -- cnexp gates, a calcium pool, a calcium-activated
channel; tests/golden/mod_kinetic -- KINETIC schemes with CONSERVE,
STEADYSTATE and a source term; tests/golden/mod_table -- a FUNCTION_TABLE
time constant) running whole spiking cells on the GPU in FP64, against an
FP64 numpy statement of the same run: the channels' numpy statements (the
ones tests/test_nmodl*.py pin the generated code to, node by node, on the
CPU) inside the FP64 oracle's step (tests/helpers.numpy_cell_run, the step
of oracle/oracle.c).  Neither side shares code with the other.

Bound: max |dV| <= 1e-5 mV over the whole trace, spikes included (the bound
of the FP64 kernel against the FP64 oracle, tests/test_gpu_parity.py)."""
import numpy as np
import pytest

from helpers import numpy_cell_run
from test_nmodl import DEMO_CELSIUS, DEMO_REV, MOD_DIR, _demo, _demo_numpy, _demo_workload, _sim
from test_nmodl_kinetic import KIN_DIR, _mixed_workload, _numpy_node
from test_nmodl_table import TABLES, TAB_DIR, _table_workload
from test_nmodl_table import _numpy as _tab_numpy

TOL_FP64_MV = 1e-5
DEMO = ("cahi", "capool", "hhdemo", "kcaf", "pas")   # _demo_numpy's mechanisms, in its state order
KIN = ("kchain", "kinsrc", "nacycle")                 # _numpy_node's, in its state order
ROWS = {"cahi": 2, "capool": 2, "hhdemo": 3, "kcaf": 1, "pas": 0, "kchain": 3, "kinsrc": 2, "nacycle": 4,
        "ktab": 1}


def node_statement(g, cell, pset):
    """node_fn for numpy_cell_run: node i runs the numpy statements of the
    mechanisms its mask holds, with its section's parameters from pset
    [n_params, n_sections] (the float32 values the GPU reads)."""
    mask = np.asarray(cell.mech_mask)
    sec = np.asarray(cell.section)
    pset = np.asarray(pset, dtype=np.float64)

    def prm_list(i, k):
        return [float(pset[p, sec[i]]) for p in g.mech_params[g.mech_index(k)]]

    def prm_dict(i, k):
        return {g.params[p][:-len(k) - 1]: float(pset[p, sec[i]]) for p in g.mech_params[g.mech_index(k)]}

    def fn(i, init, v, dt, st):
        on = [k for j, k in enumerate(g.mechs) if mask[j, i]]
        unknown = set(on) - set(DEMO) - set(KIN) - {"ktab"}
        assert not unknown, unknown
        st = dict(st or {})
        cur = cond = 0.0
        demo = [k for k in DEMO if k in on]
        if demo:
            x = np.concatenate([np.asarray(st.get(k, np.zeros(ROWS[k])), dtype=np.float64) for k in demo] or [[]])
            s, i1, g1 = _demo_numpy(demo, init, v, dt, x, {k: prm_list(i, k) for k in demo})
            r = 0
            for k in demo:
                st[k] = s[r:r + ROWS[k]]
                r += ROWS[k]
            cur, cond = cur + i1, cond + g1
        kin = [k for k in KIN if k in on]
        if kin:
            x = np.concatenate([np.asarray(st.get(k, np.zeros(ROWS[k])), dtype=np.float64) for k in kin])
            s, i2, g2 = _numpy_node(kin, init, v, dt, x, {k: prm_dict(i, k) for k in kin})
            r = 0
            for k in kin:
                st[k] = s[r:r + ROWS[k]]
                r += ROWS[k]
            cur, cond = cur + i2, cond + g2
        if "ktab" in on:
            n0 = 0.0 if init else float(st["ktab"][0])
            n, i3, g3 = _tab_numpy(init, v, dt, n0, prm_list(i, "ktab")[0])
            st["ktab"] = np.array([n])
            cur, cond = cur + i3, cond + g3
        return st, cur, cond

    return fn


def _compare(w, g, sets=(0,)):
    v64, bad = _sim(w, "fp64")
    assert bad == 0
    worst, n_spk = 0.0, 0
    for s in sets:
        for k in range(w.n_stim):
            ref = numpy_cell_run(w.cell, w.amps[k], w.dts, w.stim_node, w.stim_area, w.rec_nodes, w.v_init,
                                 node_statement(g, w.cell, w.params[s]))
            worst = max(worst, float(np.max(np.abs(v64[s, k] - ref))))
            n_spk += int(((ref[0, :-1] < -20) & (ref[0, 1:] >= -20)).sum())
    return worst, n_spk


@pytest.mark.gpu
def test_demo_set_fp64_matches_numpy_cell(ngpu_built):
    g = _demo().register()
    w = _demo_workload(g, n_sets=2, t_stop=40.0)
    worst, n_spk = _compare(w, g)
    print(f"demo set, FP64 GPU vs numpy cell: max |dV| {worst:.2e} mV, {n_spk} spikes")
    assert n_spk > 0 and worst <= TOL_FP64_MV


@pytest.mark.gpu
def test_kinetic_set_fp64_matches_numpy_cell(ngpu_built):
    from neurogpu_b200 import nmodl
    w = _mixed_workload(n_sets=2, t_stop=40.0)
    mods = sorted(MOD_DIR.glob("*.mod")) + sorted(KIN_DIR.glob("*.mod"))
    g = nmodl.generate_from_files(mods, name="demo_kin", celsius=DEMO_CELSIUS, reversal=DEMO_REV)
    worst, n_spk = _compare(w, g)
    print(f"kinetic set, FP64 GPU vs numpy cell: max |dV| {worst:.2e} mV, {n_spk} spikes")
    assert n_spk > 0 and worst <= TOL_FP64_MV


@pytest.mark.gpu
def test_table_set_fp64_matches_numpy_cell(ngpu_built):
    w, g = _table_workload(n_sets=2, t_stop=40.0)
    worst, n_spk = _compare(w, g)
    print(f"table set, FP64 GPU vs numpy cell: max |dV| {worst:.2e} mV, {n_spk} spikes")
    assert n_spk > 0 and worst <= TOL_FP64_MV
