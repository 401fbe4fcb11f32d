"""FUNCTION_TABLE in the NMODL generator (neurogpu_b200/nmodl.py).

The demo channel (tests/golden/mod_table/ktab.mod, written for these tests)
takes its time constant from a FUNCTION_TABLE of the voltage; the values are
given to the generator, as NEURON takes them from hoc.  The generated code,
compiled for the host in FP64, is checked against numpy (numpy.interp: linear
between the points, the end values outside them), on the grid, between grid
points and beyond both ends; NVRTC builds it for sm_100a; the errors for
missing or malformed tables; on the GPU, a spiking cell with the table
channel runs in FP32 against FP64."""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error
from test_nmodl import DEMO_CELSIUS, DEMO_REV, MOD_DIR, _host_lib, _run_gen, _sim

TAB_DIR = Path(__file__).resolve().parent / "golden" / "mod_table"
XS = np.linspace(-100.0, 50.0, 16)
YS = 1.0 + 4.0 * np.exp(-((XS + 40.0) / 30.0) ** 2)
TABLES = {"ktab": {"tautab": (XS, YS)}}


def _tab():
    from neurogpu_b200 import nmodl
    return nmodl.generate_from_files(sorted(TAB_DIR.glob("*.mod")), name="tab", celsius=DEMO_CELSIUS,
                                     reversal=DEMO_REV, tables=TABLES)


def _numpy(init, v, dt, n0, gbar):
    ninf = 1.0 / (1.0 + math.exp(-(v + 40.0) / 10.0))
    tau = float(np.interp(v, XS, YS))
    n = ninf if init else n0 + (-math.expm1(-dt / tau)) * (ninf - n0)
    g = gbar * n * n
    return n, g * (v - DEMO_REV["k"]), g


@pytest.mark.parametrize("init", [True, False])
def test_table_channel_matches_numpy(tmp_path, init):
    g = _tab()
    assert g.mechs == ("ktab", "pas") and g.state_rows == (1, 0)
    L = _host_lib(g, tmp_path / "tab")
    rng = np.random.default_rng(2)
    gbar = float(np.float32(0.02))
    vs = np.concatenate([XS, XS[:-1] + 3.7, [-150.0, -100.0, 50.0, 80.0, -40.0]])
    for v in vs:
        for dt in (0.025, 0.5):
            st = np.zeros((1, 32))
            st[0, 0] = rng.uniform(0.0, 1.0)
            pr = np.zeros((1, 32), dtype=np.float32)
            pr[0, 0] = gbar
            s_gen, I_gen, G_gen = _run_gen(L, init, 1, float(v), dt, st, pr)
            n, I, G = _numpy(init, float(v), dt, st[0, 0], gbar)
            assert s_gen[0] == pytest.approx(n, rel=1e-12, abs=1e-15), v
            assert I_gen == pytest.approx(I, rel=1e-12, abs=1e-15), v
            assert G_gen == pytest.approx(G, rel=1e-12, abs=1e-15), v


def test_table_set_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch):
    from neurogpu_b200 import _ffi
    g = _tab().register()
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    masks = np.array([0b11, 0b10], dtype=np.uint32)
    for precision in (0, 1):
        assert L.ngpu_jit_build(g.id, precision, masks.ctypes.data, len(masks), 10, 0, C.byref(n)) == 0, \
            L.ngpu_last_error()
        assert n.value > 0


def test_table_errors():
    from neurogpu_b200 import nmodl
    text = (TAB_DIR / "ktab.mod").read_text()
    with pytest.raises(nmodl.NmodlError, match="needs its values"):
        nmodl.generate({"ktab": text}, reversal=DEMO_REV)
    with pytest.raises(nmodl.NmodlError, match="strictly increasing"):
        nmodl.generate({"ktab": text}, reversal=DEMO_REV, tables={"ktab": {"tautab": (XS[::-1], YS)}})
    with pytest.raises(nmodl.NmodlError, match="one length"):
        nmodl.generate({"ktab": text}, reversal=DEMO_REV, tables={"ktab": {"tautab": (XS, YS[:-1])}})
    two = "NEURON { SUFFIX q }\nFUNCTION_TABLE f(a, b)\n"
    with pytest.raises(nmodl.NmodlError, match="one argument"):
        nmodl.generate({"q": two})
    # the membrane conductance is dI/dv: a table of v inside BREAKPOINT has no derivative here
    bp = ("NEURON { SUFFIX q NONSPECIFIC_CURRENT i }\nASSIGNED { v i }\nFUNCTION_TABLE f(v)\n"
          "BREAKPOINT { i = f(v) }\n")
    with pytest.raises(nmodl.NmodlError, match="differentiate"):
        nmodl.generate({"q": bp}, tables={"q": {"f": (XS, YS)}})


def _table_workload(n_sets=8, t_stop=60.0, dt=0.025):
    """A cell with the HH demo channels and the table channel (soma: hhdemo,
    ktab, pas; dendrites: ktab, pas; axon: hhdemo, pas)."""
    from neurogpu_b200 import configs, nmodl
    from neurogpu_b200.model import build_model
    mods = sorted(MOD_DIR.glob("*.mod")) + sorted(TAB_DIR.glob("*.mod"))
    g = nmodl.generate_from_files(mods, name="demo_tab", celsius=DEMO_CELSIUS, reversal=DEMO_REV,
                                  tables=TABLES).register()
    rng = np.random.default_rng(6)
    secs = configs.hh_morphology(rng, 120)
    mechs = {"soma": ("hhdemo", "ktab", "pas"), "dend": ("ktab", "pas"), "axon": ("hhdemo", "pas")}
    cell = build_model(secs, g, ("soma", "dend", "axon"), mechs, ra=100.0,
                       cm_of_region={"soma": 1.0, "dend": 1.0, "axon": 1.0})
    base = np.array(g.param_defaults, dtype=np.float64)
    base[g.param_index("g_pas")] = 3e-4
    base[g.param_index("e_pas")] = -65.0
    base[g.param_index("gbar_ktab")] = 0.005
    mult = np.exp(rng.uniform(np.log(0.7), np.log(1.4), (n_sets, 1)))
    params = np.broadcast_to(base[None, :, None], (n_sets, g.n_params, cell.n_sections)).copy()
    params[:, g.param_index("gnabar_hhdemo"), :] *= mult
    nt = int(round(t_stop / dt))
    amps = configs.step_amps([0.3, 0.8], nt, dt, 5.0, 50.0)
    return configs.Workload("demo_tab", cell, params.astype(np.float32), amps, dt, 0, float(cell.area[0]),
                            np.array([0], dtype=np.int32), -65.0), g


@pytest.mark.gpu
def test_table_channel_runs_fp32_against_fp64(ngpu_built):
    """A spiking cell with the HH demo channels and the table channel, FP32
    against FP64 within the parity bounds."""
    w, _ = _table_workload()
    v32, bad32 = _sim(w, "fp32")
    v64, bad64 = _sim(w, "fp64")
    assert bad32 == 0 and bad64 == 0
    n_spk = int(((v64[..., :-1] < -20) & (v64[..., 1:] >= -20)).sum())
    err, mism = spike_time_error(v32, v64, w.dt)
    sub = subthreshold_error(v32, v64, w.dt)
    print(f"table demo set: {n_spk} spikes; FP32 vs FP64 spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert n_spk > 0 and mism == 0 and err <= 0.05 and sub <= 0.1
