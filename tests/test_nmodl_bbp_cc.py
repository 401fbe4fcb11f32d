"""The generator on the reference's BBP cortical-cell channel set
(Figures/Figure2_BBP_CC: the TTPC channels plus a high-voltage calcium
channel `Ca` and the delayed-rectifier `KdShu2007`), where the reference tree
is present (this container, not the GPU box).

The two channels the TTPC set does not have are checked, compiled for the
host in FP64, against numpy statements of their .mod files (Ca.mod rates();
KdShu2007.mod trates(), with its ek a PARAMETER, not an ion read), to 1e-9
relative: the generator writes (-27 - v) / (exp((-27 - v)/3.8) - 1) as efun
with its series near 0, and the .mod's own nudge v += 1e-4 at v = -27 holds
for the rates only, as in NEURON.  The whole 14-mechanism set has the
mechanism order, parameter indices and state rows of the reference's own
build of the model (CParsed/AllModels.cuh), and NVRTC builds it for
sm_100a."""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

from test_nmodl import REF, _host_lib, _run_gen

CC_MODS = REF / "Figures" / "Figure2_BBP_CC"
ECA = 132.4579341637009
pytestmark = pytest.mark.skipif(not CC_MODS.exists(), reason="the reference's .mod files are not present")


def _gen(files):
    from neurogpu_b200 import nmodl
    return nmodl.generate_from_files(files, name="bbp_cc", celsius=34.0,
                                     reversal={"na": 50.0, "k": -85.0, "ca": ECA})


def _cnexp(x, xinf, tau, dt):
    return x + (-math.expm1(-dt / tau)) * (xinf - x)


def _ca_rates(v):   # Ca.mod PROCEDURE rates()
    if v == -27.0:
        v = v + 0.0001
    ma = 0.055 * (-27.0 - v) / (math.exp((-27.0 - v) / 3.8) - 1.0)
    mb = 0.94 * math.exp((-75.0 - v) / 17.0)
    ha = 0.000457 * math.exp((-13.0 - v) / 50.0)
    hb = 0.0065 / (math.exp((-v - 15.0) / 28.0) + 1.0)
    return ma / (ma + mb), 1.0 / (ma + mb), ha / (ha + hb), 1.0 / (ha + hb)


def _kd_rates(v, vhalfm, km, vhalfh, kh):   # KdShu2007.mod PROCEDURE trates(v)
    return 1.0 - 1.0 / (1.0 + math.exp((v - vhalfm) / km)), 0.6, 1.0 / (1.0 + math.exp((v - vhalfh) / kh)), 1500.0


def test_ca_and_kdshu2007_match_numpy(tmp_path):
    g = _gen([CC_MODS / "Ca.mod", CC_MODS / "KdShu2007.mod"])
    assert g.mechs == ("Ca", "KdShu2007", "pas") and g.state_rows == (2, 2, 0)
    assert g.params[:8] == ("gCabar_Ca", "gkbar_KdShu2007", "ek_KdShu2007", "vhalfm_KdShu2007", "km_KdShu2007",
                            "vhalfh_KdShu2007", "kh_KdShu2007", "q10_KdShu2007")
    L = _host_lib(g, tmp_path / "cc")
    rng = np.random.default_rng(12)
    vs = np.concatenate([np.linspace(-110.0, 50.0, 33), [-27.0, -27.02, -26.99, -43.0, -67.0]])
    for mask in (0b001, 0b010, 0b011):
        for v in vs:
            for init in (True, False):
                p = np.float32([rng.uniform(1e-5, 1e-3), rng.uniform(0.01, 0.2), -100.0, -43.0, 8.0, -67.0, 7.3, 2.3])
                rows = ([0] if mask & 1 else []) + (list(range(1, 8)) if mask & 2 else [])
                pr = np.zeros((max(len(rows), 1), 32), dtype=np.float32)
                pr[:len(rows), 0] = p[rows]
                p = p.astype(np.float64)
                st = np.zeros((4, 32))
                st[:, 0] = rng.uniform(0.0, 1.0, 4)
                dt = float(rng.choice([0.025, 0.1]))
                s_gen, I_gen, G_gen = _run_gen(L, init, mask, float(v), dt, st, pr)
                want, I, G, r = [], 0.0, 0.0, 0
                if mask & 1:
                    mi, mt, hi, ht = _ca_rates(float(v))
                    m = mi if init else _cnexp(st[r, 0], mi, mt, dt)
                    h = hi if init else _cnexp(st[r + 1, 0], hi, ht, dt)
                    want += [m, h]
                    gx = p[0] * m * m * h
                    I, G, r = I + gx * (v - ECA), G + gx, r + 2
                if mask & 2:
                    mi, mt, hi, ht = _kd_rates(float(v), *p[3:7])
                    m = mi if init else _cnexp(st[r, 0], mi, mt, dt)
                    h = hi if init else _cnexp(st[r + 1, 0], hi, ht, dt)
                    want += [m, h]
                    gx = p[1] * m * h
                    I, G = I + gx * (v - p[2]), G + gx
                np.testing.assert_allclose(s_gen[:len(want)], want, rtol=1e-9, atol=1e-15, err_msg=f"{mask} {v}")
                assert I_gen == pytest.approx(I, rel=1e-9, abs=1e-15), (mask, v, init)
                assert G_gen == pytest.approx(G, rel=1e-9, abs=1e-15), (mask, v, init)


def test_whole_cc_set_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch):
    from neurogpu_b200 import _ffi
    g = _gen(sorted(p for p in CC_MODS.glob("*.mod") if p.stem != "branching"))
    assert g.n_mech == 14 and "KdShu2007" in g.mechs and "Ca" in g.mechs
    g = g.register()
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    full = (1 << g.n_mech) - 1
    masks = np.array([full, 1 << g.mech_index("pas"), full & ~(1 << g.mech_index("Ca"))], dtype=np.uint32)
    assert L.ngpu_jit_build(g.id, 0, masks.ctypes.data, len(masks), 10, 0, C.byref(n)) == 0, L.ngpu_last_error()
    assert n.value > 0


def test_cc_set_layout_matches_reference_build():
    """Mechanism order, parameter indices and channel-state rows of the
    generated set against the reference's own build of this model
    (CParsed/AllModels.cuh CALL_TO_BREAK_CU: CuBreakpointModel_<mech>(...,
    state_macro(s, ...), param_macro(p, ...), ...)); the calcium pool keeps
    cai in its own array there and in two state rows (cai, ica) here."""
    import re
    g = _gen(sorted(p for p in CC_MODS.glob("*.mod") if p.stem != "branching"))
    text = (CC_MODS / "CParsed" / "AllModels.cuh").read_text()
    line = next(ln for ln in text.splitlines() if ln.startswith("#define CALL_TO_BREAK_CU"))
    calls = re.findall(r"CuBreakpointModel_(\w+)\(([^;]*?)\);", line)
    assert tuple(name for name, _ in calls) == g.mechs
    for k, (name, args) in enumerate(calls):
        params = tuple(int(i) for i in re.findall(r"param_macro\((\d+),", args))
        assert params == tuple(g.mech_params[k]), name
        states = re.findall(r"state_macro\((\d+),", args)
        assert len(states) == (g.state_rows[k] if name != "CaDynamics_E2" else 0), name
    assert g.n_params == 1 + max(max(p) for p in g.mech_params if p)


def test_cc_data_dir_reads_with_the_generated_set():
    """The reference's own input files for this model (Data/: 224 nodes in
    103 compartments, 14 boolModel rows, 26 parameters per compartment) read
    with the generated set: its mechanism masks are the file's boolModel
    rows and its parameters the file's, unpermuted.  A set whose sizes do
    not match the files is refused."""
    from neurogpu_b200 import formats
    g = _gen(sorted(p for p in CC_MODS.glob("*.mod") if p.stem != "branching"))
    data = CC_MODS / "Data"
    m = formats.read_data_dir(data, mechset=g)
    c = m.cell
    assert c.mechset is g and c.n_nodes == 224 and c.n_sections == 103
    bc = m.raw["basic_const"]
    np.testing.assert_array_equal(c.mech_mask, (bc["boolModel"].reshape(14, 224) != 0).astype(np.uint8))
    assert m.params.shape[1:] == (26, 103) and m.params is m.raw["file_params"]
    assert c.mech_mask.any(axis=1).all()     # every mechanism on some node
    with pytest.raises(ValueError, match="mechanisms"):
        formats.read_data_dir(data, mechset=_gen([CC_MODS / "Ca.mod"]))
    with pytest.raises(ValueError, match="no library mechanism set"):
        formats.read_data_dir(data)


def test_cc_basic_const_regenerates_byte_for_byte(tmp_path):
    """The reference's BasicConstSegP.csv of this model (224 nodes), read with
    the generated set into a CellModel and written again: the same bytes;
    the whole Data/ directory written and read back with the set."""
    from neurogpu_b200 import formats
    g = _gen(sorted(p for p in CC_MODS.glob("*.mod") if p.stem != "branching"))
    data = CC_MODS / "Data"
    r = formats.read_data_dir(data, mechset=g)
    bm = r.raw["basic_const"]["boolModel"].reshape(14, -1)
    out = tmp_path / "BasicConstSegP.csv"
    formats.write_basic_const_segp(out, r.cell, bm)
    assert out.read_text() == (data / "BasicConstSegP.csv").read_text()
    d2 = tmp_path / "Data"
    formats.write_data_dir(d2, r.cell, r.params, r.amps, r.dts, r.stim_node, r.stim_area, r.rec_nodes, r.v_init,
                           0.025, bool_model=bm)
    s = formats.read_data_dir(d2, mechset=g)
    for k in ("parent", "a", "b", "mech_mask", "section", "cm"):
        np.testing.assert_array_equal(getattr(s.cell, k), getattr(r.cell, k), err_msg=k)
    np.testing.assert_allclose(s.params, r.params, rtol=5e-6, atol=0)   # AllParams.csv: %.5E
    np.testing.assert_array_equal(s.amps, r.amps)
    np.testing.assert_array_equal(s.dts, r.dts)
