"""The reference-format writers of neurogpu_b200.formats: BasicConstSegP.csv
regenerated from a model byte for byte, and whole Data/ directories written and
read back."""
from pathlib import Path

import numpy as np
import pytest

from neurogpu_b200 import configs
from neurogpu_b200 import formats as F
from neurogpu_b200.model import CellModel

GOLDEN = Path(__file__).parent / "golden"
SHIPPED = {
    "ttpc512": dict(stim_index=0, params_file="AllParams_reference.csv"),
    "mainen384": {},
    "passive384": {},
}


def _bool_model(bc):
    return bc["boolModel"].reshape(int(bc["NModels"][0]), -1)


@pytest.mark.parametrize("name", sorted(SHIPPED))
def test_fields_regenerate_the_shipped_file(name):
    """Every field the reference's auxiliary-data builder derives (level
    schedule, father rows, ancestor table, 32-wide level rows) recomputed from
    the file's own Ks / e / f / SegToComp / Cms / boolModel: the same text."""
    path = GOLDEN / name / "BasicConstSegP.csv"
    bc = F.read_basic_const_segp(path)
    fields = F.basic_const_fields(bc["Ks"].astype(np.int64), bc["e"], bc["f"], bc["SegToComp"], bc["Cms"],
                                  _bool_model(bc), int(bc["NComps"][0]))
    bad = [k for k in F.BCS_FIELDS if not np.array_equal(np.asarray(fields[k]).reshape(-1), bc[k])]
    assert bad == []
    assert F.format_basic_const_segp(fields) == path.read_text()


@pytest.mark.parametrize("name", sorted(SHIPPED))
def test_cell_writes_the_shipped_file(name, tmp_path):
    """A CellModel read from the file and written again: the same bytes."""
    r = F.read_data_dir(GOLDEN / name, **SHIPPED[name])
    out = tmp_path / "BasicConstSegP.csv"
    F.write_basic_const_segp(out, r.cell, _bool_model(r.raw["basic_const"]))
    assert out.read_text() == (GOLDEN / name / "BasicConstSegP.csv").read_text()


def _same_cell(c1: CellModel, c2: CellModel):
    for k in ("parent", "a", "b", "mech_mask", "section", "cm"):
        np.testing.assert_array_equal(getattr(c1, k), getattr(c2, k), err_msg=k)
    assert c1.n_sections == c2.n_sections and c1.mechset.name == c2.mechset.name


@pytest.mark.parametrize("name", sorted(SHIPPED))
def test_data_dir_round_trip(name, tmp_path):
    r = F.read_data_dir(GOLDEN / name, **SHIPPED[name])
    _, _, pmap = F.mechset_for(int(r.raw["basic_const"]["NModels"][0]), r.raw["file_params"].shape[1])
    stim = SHIPPED[name].get("stim_index")
    F.write_data_dir(tmp_path, r.cell, r.params, r.amps, r.dts, r.stim_node, r.stim_area, r.rec_nodes, r.v_init,
                     0.025, bool_model=_bool_model(r.raw["basic_const"]), stim_index=stim, param_index=pmap)
    s = F.read_data_dir(tmp_path, stim_index=stim)
    _same_cell(r.cell, s.cell)
    # AllParams.csv holds 6 significant digits (%.5E)
    np.testing.assert_allclose(s.params, r.params, rtol=5e-6, atol=0)
    np.testing.assert_array_equal(s.amps, r.amps)
    np.testing.assert_array_equal(s.dts, r.dts)
    np.testing.assert_array_equal(s.rec_nodes, r.rec_nodes)
    assert (s.stim_node, s.stim_area, s.v_init) == (r.stim_node, r.stim_area, r.v_init)


def _one_child_root(n_comp=96, seed=3) -> CellModel:
    """A random binary cable under a root with one child (the reference's
    format counts the root as its own first child, so a root may carry one
    more)."""
    rng = np.random.default_rng(seed)
    p0, length, diam = configs.random_binary_cable(rng, n_comp, 20.0, (1.0, 4.0))
    parent = np.concatenate([[-1], np.where(p0 < 0, 0, p0 + 1)]).astype(np.int32)
    length = np.concatenate([[10.0], length])
    diam = np.concatenate([[10.0], diam])
    a, b, area = configs.cable_coefficients(parent, length, diam, 100.0)
    n = parent.size
    ms = configs.TTPC
    mask = np.zeros((ms.n_mech, n), dtype=np.uint8)
    mask[ms.mech_index("pas")] = 1
    mask[ms.mech_index("NaTa_t"), : n // 3] = 1
    sec = (np.arange(n) * 7 // n).astype(np.int32)
    cell = CellModel(parent=parent, a=a, b=b, cm=np.linspace(0.8, 1.2, n), section=sec, n_sections=7, mechset=ms,
                     mech_mask=mask, area=area)
    cell.validate()
    return cell


def test_synthetic_model_round_trip(tmp_path):
    cell = _one_child_root()
    rng = np.random.default_rng(0)
    ms = cell.mechset
    params = rng.uniform(0.5, 2.0, (3, ms.n_params, cell.n_sections)).astype(np.float32)
    amps = np.zeros((2, 400), dtype=np.float32)
    amps[:, 100:300] = [[0.2], [0.5]]
    dts = np.full(400, 0.025, dtype=np.float32)
    F.write_data_dir(tmp_path, cell, params, amps, dts, stim_node=0, stim_area=float(np.float32(cell.area[0])),
                     rec_nodes=[0, 5], v_init=-65.0, dt=0.025)
    s = F.read_data_dir(tmp_path)
    # the reader zeroes the root's coupling; the written tree is the same
    want_a, want_b = cell.a.copy(), cell.b.copy()
    want_a[0] = want_b[0] = 0.0
    np.testing.assert_array_equal(s.cell.parent, cell.parent)
    # BasicConstSegP.csv prints every value with 9 decimals
    np.testing.assert_allclose(s.cell.a, want_a, rtol=0, atol=5.0001e-10)
    np.testing.assert_allclose(s.cell.b, want_b, rtol=0, atol=5.0001e-10)
    np.testing.assert_allclose(s.cell.cm, cell.cm, rtol=0, atol=5.0001e-10)
    np.testing.assert_array_equal(s.cell.mech_mask, cell.mech_mask)
    np.testing.assert_array_equal(s.cell.section, cell.section)
    np.testing.assert_allclose(s.params, params, rtol=5e-6)
    np.testing.assert_array_equal(s.amps, amps)
    assert list(s.rec_nodes) == [0, 5] and s.v_init == -65.0 and s.stim_node == 0
    bc = s.raw["basic_const"]
    assert int(bc["Depth"][0]) >= 1 and int(bc["N"][0]) == cell.n_nodes
    # writing the model read back gives the same file again
    again = tmp_path / "again.csv"
    F.write_basic_const_segp(again, s.cell, _bool_model(bc))
    assert again.read_text() == (tmp_path / "BasicConstSegP.csv").read_text()


def test_root_with_two_children_is_rejected(tmp_path):
    """A root with two children, or any node with three, does not fit the
    reference's two-child solver."""
    w = configs.passive_cable(n_sets=2, t_stop=1.0)
    with pytest.raises(ValueError, match="more than two children"):
        F.write_basic_const_segp(tmp_path / "x.csv", w.cell)



from oracle_py import REFERENCE_DIR as REF
# parameters of the built-in sets' reference builds, by boolModel row count
BUILT_IN_PARAMS = {13: 19, 7: 34, 1: 2}      # TTPC, Mainen, single-mechanism passive


def _shipped_models():
    if not REF.exists():
        return []
    return sorted(str(p.parent.relative_to(REF)) for p in REF.rglob("Data/BasicConstSegP.csv")
                  if not p.is_relative_to(REF / "Code") and "CoreNeuron" not in p.parts)


@pytest.mark.skipif(not REF.exists(), reason="the reference tree is not present")
@pytest.mark.parametrize("sub", _shipped_models())
def test_every_shipped_model_regenerates(sub, tmp_path):
    """Every model Data/ directory of the reference tree (outside the bare
    Code/ snapshots, which ship no parameter files): its BasicConstSegP.csv,
    read into a CellModel with the mechanism set of its build (built-in, or
    generated from the model's own .mod files) and written again, is the same
    text.  Parameters are not read here: Figure4_DEAP's AllParams rows (the
    GA's scratch output) hold 4577-4578 of the build's 19 x 241 values."""
    from neurogpu_b200 import nmodl
    d = REF / sub
    bc = F.read_basic_const_segp(d / "BasicConstSegP.csv")
    nm = int(bc["NModels"][0])
    ms = None
    n_params = BUILT_IN_PARAMS.get(nm)
    if n_params is None:
        mods = sorted(q for q in d.parent.glob("*.mod") if q.stem != "branching")
        ms = nmodl.generate_from_files(mods, name="shipped", celsius=34.0,
                                       reversal={"na": 50.0, "k": -85.0, "ca": 132.458})
        n_params = ms.n_params
    cell = F.cell_from_basic_const(bc, n_params, ms)
    out = tmp_path / "BasicConstSegP.csv"
    F.write_basic_const_segp(out, cell, _bool_model(bc))
    assert out.read_text() == (d / "BasicConstSegP.csv").read_text()
