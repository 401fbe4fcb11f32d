"""Pins of the CPU oracle (and of the reference-format readers) against the
reference's own artefacts -- no GPU needed.

* channels_{ttpc,mainen}.npz: the reference's generated channel functions
  (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cu,
  Figures/FigureS4_mainen/CParsed/AllModels.cu), compiled for the host from
  the reference's sources and evaluated on a seeded grid by
  tests/golden/make_golden.py.  The oracle's node functions must reproduce
  them mechanism by mechanism (the reference stores FP32, computes in FP64).
* BasicConstSegP.csv of three shipped models: the parent vector the readers
  derive from Ks must regenerate the reference's own SonNoVec and FIdxs
  tables (NeuroGPU_Base/scripts/pyscripts/create_auxilliary_data_3.py:53-84).
* Fmatrix.csv: e and f are the reversed B and A columns
  (create_auxilliary_data_3.py:316-321).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def _oracle_node(oracle, ms, mech, what, v, dt, s_in, p, n_states, n_mech):
    L = oracle.lib()
    mask = np.zeros(n_mech, dtype=np.uint8)
    mask[mech] = 1
    s = s_in.astype(np.float64).copy()
    pd = p.astype(np.float64)
    g = C.c_double(0.0)
    I = 0.0
    if what == 0:
        L.ong_node_init_f64(ms, mask.ctypes.data, float(v), pd.ctypes.data, s.ctypes.data)
    elif what == 1:
        L.ong_node_deriv_f64(ms, mask.ctypes.data, float(dt), float(v), pd.ctypes.data, s.ctypes.data)
    else:
        I = L.ong_node_current_f64(ms, mask.ctypes.data, float(v), pd.ctypes.data, s.ctypes.data, C.byref(g))
    return s, I, g.value


@pytest.mark.parametrize("name,ms,n_states,n_mech", [("ttpc", 0, 19, 13), ("mainen", 1, 8, 9)])
def test_oracle_channels_match_reference_build(oracle, name, ms, n_states, n_mech):
    z = np.load(GOLD / f"channels_{name}.npz")
    worst = 0.0
    for k in range(z["mech"].size):
        mech, what = int(z["mech"][k]), int(z["what"][k])
        s, I, g = _oracle_node(oracle, ms, mech, what, z["v"][k], z["dt"][k], z["s_in"][k], z["p"][k],
                               n_states, n_mech)
        ref_s = z["s_out"][k].astype(np.float64)
        # states, cai and ica (eca is carried as a float by the reference: compare loosely)
        idx = list(range(n_states)) + [n_states, n_states + 2]
        np.testing.assert_allclose(s[idx], ref_s[idx], rtol=2e-6, atol=1e-9,
                                   err_msg=f"{name} mech {mech} what {what} v {z['v'][k]}")
        np.testing.assert_allclose(s[n_states + 1], ref_s[n_states + 1], rtol=1e-5)
        if what == 2:
            np.testing.assert_allclose(I, z["I"][k], rtol=2e-6, atol=1e-9,
                                       err_msg=f"{name} mech {mech} current v {z['v'][k]}")
            if name == "ttpc":  # the TTPC breakpoints' summed conductance is dI/dv
                np.testing.assert_allclose(g, z["G"][k], rtol=2e-6, atol=1e-9)
        rel = np.abs(s[idx] - ref_s[idx]) / np.maximum(1.0, np.abs(ref_s[idx]))
        worst = max(worst, float(rel.max()))
    assert worst < 1e-6     # a few FP32 ulps of the reference's stored outputs


@pytest.mark.parametrize("model", ["ttpc512", "mainen384", "passive384"])
def test_topology_known_answers(model):
    from neurogpu_b200 import formats
    bc = formats.read_basic_const_segp(GOLD / model / "BasicConstSegP.csv")
    parent = formats.parent_from_ks(bc["Ks"])
    n = int(bc["N"][0])
    assert parent[0] == -1 and np.all(parent[1:] < np.arange(1, n))
    assert np.array_equal(formats.son_no_vec(parent), bc["SonNoVec"].astype(np.int64))
    tab = formats.ancestor_table(bc["Ks"])
    assert tab.shape[0] == int(bc["LognDepth"][0])
    assert np.array_equal(tab.reshape(-1), bc["FIdxs"].astype(np.int64))


@pytest.mark.parametrize("model", ["mainen384", "passive384"])
def test_coefficients_are_reversed_fmatrix_columns(model):
    from neurogpu_b200 import formats
    bc = formats.read_basic_const_segp(GOLD / model / "BasicConstSegP.csv")
    fm = np.loadtxt(GOLD / model / "Fmatrix.csv")
    np.testing.assert_allclose(bc["f"], fm[::-1, 1], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(bc["e"], fm[::-1, 2], rtol=1e-7, atol=1e-9)


@pytest.mark.parametrize("model,mechset,n_params", [("ttpc512", "ttpc", 19), ("mainen384", "mainen", 34),
                                                    ("passive384", "ttpc", 19)])
def test_reference_data_dirs_read(model, mechset, n_params):
    from neurogpu_b200 import formats
    pf = "AllParams_reference.csv" if model == "ttpc512" else None
    m = formats.read_data_dir(GOLD / model, stim_index=0 if model == "ttpc512" else None, params_file=pf)
    assert m.cell.mechset.name == mechset
    assert m.params.shape == (1, n_params, m.cell.n_sections)
    assert m.amps.shape[1] == 3168 and np.allclose(m.dts, 0.1)
    assert m.stim_node == 1 and list(m.rec_nodes) == [0]
    if model == "passive384":  # the one-mechanism build's (g, e) land on pas
        gp = m.params[0, 14]
        assert set(np.unique(gp)) <= {0.0, np.float32(0.001)}
        assert set(np.unique(m.params[0, 15])) <= {0.0, -70.0}


def test_oracle_runs_shipped_models(oracle):
    """The reference's own models run through the oracle without non-finite
    values and settle near their resting potentials before the step."""
    from neurogpu_b200 import formats
    for model, pf, sidx in (("ttpc512", "AllParams_reference.csv", 0), ("mainen384", None, None),
                            ("passive384", None, None)):
        m = formats.read_data_dir(GOLD / model, stim_index=sidx, params_file=pf)
        c = m.cell
        out = oracle.run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask,
                         m.params, m.amps[:, :400], m.dts[:400], m.stim_node, m.stim_area, m.rec_nodes,
                         m.v_init)
        assert np.all(np.isfinite(out))
        assert abs(out[0, 0, 0, 99] - m.v_init) < 15.0


def test_allparams_parse_matches_reference_parser():
    """AllParams values parse to the reference parser's float32 bits
    (src/Util.cu:143-185), which differ from a correctly rounded parse for a
    sizeable share of tokens."""
    from neurogpu_b200.formats import ref_atof
    z = np.load(GOLD / "atof_vectors.npz")
    got = np.array([ref_atof(str(t)) for t in z["tokens"]], dtype=np.float32).view(np.uint32)
    assert np.array_equal(got, z["bits"])
    rounded = np.array([np.float32(float(t)) for t in z["tokens"]], dtype=np.float32).view(np.uint32)
    assert np.count_nonzero(rounded != z["bits"]) > 0.05 * z["bits"].size
    with pytest.raises(ValueError):
        ref_atof("1.5e3")
