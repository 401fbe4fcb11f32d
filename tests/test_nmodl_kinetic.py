"""KINETIC schemes in the NMODL generator (neurogpu_b200/nmodl.py).

The demo schemes (tests/golden/mod_kinetic, written for these tests): a
three-state potassium chain and a four-state sodium cycle, both with CONSERVE
and SOLVE ... STEADYSTATE sparse in INITIAL, and a two-state scheme with a
source term and no conservation law.  The generated code, compiled for the
host in FP64, is checked against a numpy statement of backward Euler
(numpy.linalg.solve of (I - dt Q) x' = x + dt s, the conserved state's row
replaced by the conservation law), step and steady state; then the
properties a step must have (conservation, the steady state is a fixed point
of the step).  On the GPU a set mixing these schemes with the HH demo runs a
spiking cell in FP32 against FP64."""
import math
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error
from test_nmodl import DEMO_CELSIUS, DEMO_REV, MOD_DIR, _host_lib, _run_gen, _sim

KIN_DIR = Path(__file__).resolve().parent / "golden" / "mod_kinetic"
STEADY_DT = 1e9


def _kin():
    from neurogpu_b200 import nmodl
    return nmodl.generate_from_files(sorted(KIN_DIR.glob("*.mod")), name="kin", celsius=DEMO_CELSIUS,
                                     reversal=DEMO_REV)


# ------------------------------------------------ numpy statement of the schemes
def _scheme(name, v, p):
    """(states, reactions (a, b, kf, kb), sources {state: s}, conserved state or None)."""
    if name == "kchain":
        a0, b0 = p["a0"], p["b0"]
        a1, b1 = a0 * math.exp((v + 40) / 20), b0 * math.exp(-(v + 40) / 25)
        a2, b2 = 2 * a0 * math.exp((v + 30) / 15), b0 * math.exp(-(v + 30) / 30)
        return ["c1", "c2", "o"], [("c1", "c2", a1, b1), ("c2", "o", a2, b2)], {}, "o"
    if name == "nacycle":
        ao, bo = 3 * math.exp((v + 35) / 9), 0.5 * math.exp(-(v + 35) / 12)
        ai, bi = 0.8 * math.exp((v + 50) / 30), 0.02 * math.exp(-(v + 70) / 10)
        ks = p["kslow"]
        return (["c", "o", "i1", "i2"],
                [("c", "o", ao, bo), ("o", "i1", ai, 0.01 * bi), ("i1", "c", bi, 0.05 * ai),
                 ("i1", "i2", ks, 0.1 * ks)], {}, "i2")
    if name == "kinsrc":
        return ["a", "b"], [("a", "b", p["k1"] * math.exp(v / 40), p["k2"])], {"a": p["s"]}, None
    raise KeyError(name)


def _be_step(name, v, dt, x, p):
    """One backward-Euler step of a scheme from x (state order of the STATE block)."""
    states, reacts, src, cons = _scheme(name, v, p)
    n = len(states)
    ix = {s: i for i, s in enumerate(states)}
    Q = np.zeros((n, n))
    for a, b, kf, kb in reacts:
        i, j = ix[a], ix[b]
        Q[i, i] -= kf
        Q[j, i] += kf
        Q[j, j] -= kb
        Q[i, j] += kb
    A = np.eye(n) - dt * Q
    rhs = np.array(x, dtype=np.float64) + dt * np.array([src.get(s, 0.0) for s in states])
    if cons is not None:
        A[ix[cons], :] = 1.0
        rhs[ix[cons]] = 1.0
    return np.linalg.solve(A, rhs), Q


_ROWS = {"kchain": 3, "kinsrc": 2, "nacycle": 4, "pas": 0}
_PRM = {"kchain": {"gbar": 0.01, "a0": 0.2, "b0": 0.05}, "kinsrc": {"g": 0.001, "e": -20.0, "k1": 0.3, "k2": 0.1,
                                                                     "s": 0.02},
        "nacycle": {"gbar": 0.05, "kslow": 0.002}, "pas": {"g": 3e-4, "e": -68.0}}
_ORDER = ["kchain", "kinsrc", "nacycle", "pas"]


def _numpy_node(on, init, v, dt, st, prm):
    out, I, G = [], 0.0, 0.0
    r = 0
    for k in _ORDER:
        if k not in on:
            continue
        x = st[r:r + _ROWS[k]]
        r += _ROWS[k]
        p = prm[k]
        if k == "pas":
            I += p["g"] * (v - p["e"])
            G += p["g"]
            continue
        if init:
            x = [0.2, 0.1] if k == "kinsrc" else _be_step(k, v, STEADY_DT, np.zeros(_ROWS[k]), p)[0]
        else:
            x = _be_step(k, v, dt, x, p)[0]
        out += list(x)
        if k == "kchain":
            g = p["gbar"] * x[2]
            I += g * (v - DEMO_REV["k"])
        elif k == "nacycle":
            g = p["gbar"] * x[1]
            I += g * (v - DEMO_REV["na"])
        else:
            g = p["g"] * x[1]
            I += g * (v - p["e"])
        G += g
    return np.array(out), I, G


def test_layout():
    g = _kin()
    assert g.mechs == ("kchain", "kinsrc", "nacycle", "pas")
    assert g.state_rows == (3, 2, 4, 0)
    assert g.params[:3] == ("gbar_kchain", "a0_kchain", "b0_kchain")


def _inputs(g, on, rng):
    rows = sum(_ROWS[k] for k in on)
    st = np.zeros((max(rows, 1), 32))
    st[:rows, 0] = rng.uniform(0.0, 1.0, rows)
    pvals = [x for k in g.mechs if k in on for x in _PRM[k].values()]
    pr = np.zeros((max(len(pvals), 1), 32), dtype=np.float32)
    pr[:len(pvals), 0] = pvals
    prm32 = {k: {n: float(np.float32(x)) for n, x in vals.items()} for k, vals in _PRM.items()}
    mask = sum(1 << g.mech_index(k) for k in on)
    return rows, st, pr, prm32, mask


@pytest.mark.parametrize("init", [True, False])
def test_schemes_match_numpy(tmp_path, init):
    g = _kin()
    L = _host_lib(g, tmp_path / "kin")
    rng = np.random.default_rng(5)
    for on in (["kchain"], ["nacycle"], ["kinsrc"], ["kchain", "kinsrc", "nacycle", "pas"]):
        for v in np.linspace(-100.0, 40.0, 15):
            for dt in (0.025, 0.5):
                rows, st, pr, prm32, mask = _inputs(g, on, rng)
                s_gen, I_gen, G_gen = _run_gen(L, init, mask, float(v), dt, st, pr)
                s_np, I_np, G_np = _numpy_node(on, init, float(v), dt, st[:rows, 0], prm32)
                # the steady state is a solve at dt = 1e9: its conditioning costs digits
                rtol = 1e-7 if init else 1e-11
                np.testing.assert_allclose(s_gen[:rows], s_np, rtol=rtol, atol=1e-13, err_msg=f"{on} v={v}")
                assert I_gen == pytest.approx(I_np, rel=rtol, abs=1e-15), (on, v)
                assert G_gen == pytest.approx(G_np, rel=rtol, abs=1e-15), (on, v)


def test_step_properties(tmp_path):
    """A step conserves what CONSERVE names (whatever the states held
    before), keeps states in [0, 1] from a distribution, and leaves the
    steady state where it is."""
    g = _kin()
    L = _host_lib(g, tmp_path / "kin")
    rng = np.random.default_rng(11)
    for k in ("kchain", "nacycle"):
        for v in (-90.0, -60.0, -35.0, 0.0, 30.0):
            rows, st, pr, prm32, mask = _inputs(g, [k], rng)
            st[:rows, 0] /= st[:rows, 0].sum()
            s1, _, _ = _run_gen(L, False, mask, v, 0.025, st, pr)
            assert s1[:rows].sum() == pytest.approx(1.0, abs=1e-13)
            assert np.all(s1[:rows] >= -1e-15) and np.all(s1[:rows] <= 1 + 1e-15)
            ss, _, _ = _run_gen(L, True, mask, v, 0.025, st, pr)
            st2 = st.copy()
            st2[:rows, 0] = ss[:rows]
            s2, _, _ = _run_gen(L, False, mask, v, 0.025, st2, pr)
            # a 1e9 ms step stops short of the fixed point by about
            # 1 / (1e9 x the slowest rate): 1.4e-7 relative for 0.007 /ms
            _, Q = _be_step(k, v, 0.025, ss[:rows], prm32[k])
            slow = np.min(np.abs(Q[Q != 0]))
            tol = 4.0 / (STEADY_DT * slow)
            np.testing.assert_allclose(s2[:rows], ss[:rows], rtol=tol, atol=1e-14)
            assert np.max(np.abs(Q @ ss[:rows])) <= 2.0 / STEADY_DT


@pytest.mark.parametrize("text,msg", [
    ("NEURON { SUFFIX q }\nSTATE { a b c }\nBREAKPOINT { SOLVE k METHOD sparse }\n"
     "KINETIC k { ~ a + b <-> c (1, 2) }\n", "first-order"),
    ("NEURON { SUFFIX q }\nSTATE { a b }\nBREAKPOINT { SOLVE k METHOD sparse }\n"
     "KINETIC k { ~ 2 a <-> b (1, 2) }\n", "stoichiometric"),
    ("NEURON { SUFFIX q }\nSTATE { a b }\nBREAKPOINT { SOLVE k METHOD cnexp }\n"
     "KINETIC k { ~ a <-> b (1, 2) }\n", "sparse only"),
    ("NEURON { SUFFIX q }\nSTATE { a b }\nASSIGNED { z }\nBREAKPOINT { SOLVE k METHOD sparse }\n"
     "KINETIC k { ~ a <-> z (1, 2) }\n", "not a STATE"),
    ("NEURON { SUFFIX q }\nSTATE { a b }\nBREAKPOINT { SOLVE k METHOD sparse }\n"
     "KINETIC k { ~ a <-> b (1, 2) CONSERVE a*b = 1 }\n", "linear"),
    ("NEURON { SUFFIX q }\nSTATE { x }\nBREAKPOINT { SOLVE d METHOD cnexp }\nINITIAL { SOLVE d STEADYSTATE sparse }\n"
     "DERIVATIVE d { x' = -x }\n", "only KINETIC"),
])
def test_unsupported_kinetic_input_is_an_error(text, msg):
    from neurogpu_b200 import nmodl
    with pytest.raises(nmodl.NmodlError, match=msg):
        nmodl.generate({"q": text})


@pytest.mark.parametrize("precision", [0, 1])
def test_kinetic_set_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch, precision):
    import ctypes as C

    from neurogpu_b200 import _ffi
    g = _kin().register()
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    masks = np.array([0b1111, 0b0101], dtype=np.uint32)
    rc = L.ngpu_jit_build(g.id, precision, masks.ctypes.data, len(masks), 10, 0, C.byref(n))
    assert rc == 0, L.ngpu_last_error()
    assert n.value > 0


# ------------------------------------------------------------------- GPU
def _mixed_workload(n_sets=8, t_stop=60.0, dt=0.025, seed=4):
    from neurogpu_b200 import configs, nmodl
    from neurogpu_b200.model import build_model
    mods = sorted(MOD_DIR.glob("*.mod")) + sorted(KIN_DIR.glob("*.mod"))
    g = nmodl.generate_from_files(mods, name="demo_kin", celsius=DEMO_CELSIUS, reversal=DEMO_REV).register()
    rng = np.random.default_rng(seed)
    secs = configs.hh_morphology(rng, 120)
    mechs = {"soma": ("hhdemo", "kchain", "nacycle", "pas"), "dend": ("kchain", "kinsrc", "pas"),
             "axon": ("hhdemo", "nacycle", "pas")}
    cell = build_model(secs, g, ("soma", "dend", "axon"), mechs, ra=100.0,
                       cm_of_region={"soma": 1.0, "dend": 1.0, "axon": 1.0})
    base = np.array(g.param_defaults, dtype=np.float64)
    base[g.param_index("g_pas")] = 3e-4
    base[g.param_index("e_pas")] = -65.0
    base[g.param_index("gbar_nacycle")] = 0.01
    base[g.param_index("gbar_kchain")] = 0.002
    mult = np.exp(rng.uniform(np.log(0.7), np.log(1.4), (n_sets, 1)))
    params = np.broadcast_to(base[None, :, None], (n_sets, g.n_params, cell.n_sections)).copy()
    params[:, g.param_index("gnabar_hhdemo"), :] *= mult
    nt = int(round(t_stop / dt))
    amps = configs.step_amps([0.3, 0.8], nt, dt, 5.0, 50.0)
    return configs.Workload("demo_kin", cell, params.astype(np.float32), amps, dt, 0, float(cell.area[0]),
                            np.array([0], dtype=np.int32), -65.0)


@pytest.mark.gpu
def test_kinetic_set_runs_fp32_against_fp64(ngpu_built):
    w = _mixed_workload()
    v32, bad32 = _sim(w, "fp32")
    v64, bad64 = _sim(w, "fp64")
    assert bad32 == 0 and bad64 == 0
    n_spk = int(((v64[..., :-1] < -20) & (v64[..., 1:] >= -20)).sum())
    err, mism = spike_time_error(v32, v64, w.dt)
    sub = subthreshold_error(v32, v64, w.dt)
    print(f"kinetic demo set: {n_spk} spikes; FP32 vs FP64 spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert n_spk > 0
    assert mism == 0 and err <= 0.05 and sub <= 0.1
