"""NMODL -> channel code generator (neurogpu_b200/nmodl.py).

CPU checks of the generated device code, compiled for the host in FP64:
  * a demo set written for these tests (tests/golden/mod: Hodgkin-Huxley
    sodium / potassium, a calcium pool, a high-threshold calcium current, a
    calcium-activated potassium current, NEURON's pas) against a numpy
    statement of the same equations, mechanism by mechanism and together;
  * where the reference tree is present (this container, not the GPU box),
    the sets generated from the reference's own .mod files (the BBP TTPC
    channels of NeuroGPU_Base/scripts/template and the Mainen channels of
    Figures/FigureS4_mainen) against the hand-written channel code, which is
    pinned to the reference's AllModels.cu (test_oracle_pins,
    test_channels_host): same mechanism order, parameter list and row layout,
    and the same states, current and conductance to 1e-9 relative;
  * the symbolic pieces (linear form of a derivative, d/dv) and the errors
    for unsupported input;
  * NVRTC builds the runtime kernels of a defined set for sm_100a.
GPU checks (marked gpu): a defined set runs end to end (FP32 against FP64),
and a generated pas-only set reproduces the built-in TTPC pas simulation.
"""
import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error

ROOT = Path(__file__).resolve().parent.parent
MOD_DIR = ROOT / "tests" / "golden" / "mod"
from oracle_py import REFERENCE_DIR as REF
TTPC_MODS = REF / "NeuroGPU_Base" / "scripts" / "template"
MAINEN_MODS = REF / "Figures" / "FigureS4_mainen"
MAINEN_CONSTANTS = {
    "ca": {"cao": 2.5, "vshift": 0, "temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "na": {"vshift": -5, "temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "kca": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "km": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "kv": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "cad": {"depth": 0.09334562733124982, "taur": 200.0, "cainf": 1e-4},
}
DEMO_CELSIUS = 6.3
DEMO_REV = {"na": 50.0, "k": -77.0}

PROBE = r'''
#include <stdint.h>
#include "ngpu_generated.cuh"
extern "C" void probe_gen_f64(int init, uint32_t mask, double v, double dt, double* st, const float* pr,
                              double* I, double* G) {
    double i = 0, g = 0;
    if (init) ngpu::generated_node<double, true>(mask, v, dt, st, pr, i, g);
    else ngpu::generated_node<double, false>(mask, v, dt, st, pr, i, g);
    *I = i;
    *G = g;
}
'''


def _demo():
    from neurogpu_b200 import nmodl
    return nmodl.generate_from_files(sorted(MOD_DIR.glob("*.mod")), name="demo", celsius=DEMO_CELSIUS,
                                     reversal=DEMO_REV)


def _host_lib(gen, tmp: Path):
    tmp.mkdir(parents=True, exist_ok=True)
    (tmp / "ngpu_generated.cuh").write_text(gen.source)
    (tmp / "probe.cu").write_text(PROBE)
    r = subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
                        "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "neurogpu_b200" / "csrc"), "-I", str(tmp),
                        str(tmp / "probe.cu"), "-o", str(tmp / "libprobe.so")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(str(tmp / "libprobe.so"))
    L.probe_gen_f64.restype = None
    return L


def _run_gen(L, init, mask, v, dt, st, pr):
    s = st.copy()
    I, G = C.c_double(), C.c_double()
    L.probe_gen_f64(int(init), mask, C.c_double(v), C.c_double(dt), s.ctypes.data, pr.ctypes.data, C.byref(I),
                    C.byref(G))
    return s[:, 0], I.value, G.value


# --------------------------------------------------- numpy statement of the demo set
F = 96485.309


def _demo_numpy(on, init, v, dt, st, prm):
    """States (in row order), I, G of the demo mechanisms `on` (names) at one node."""
    ktf = 1000.0 * 8.3134 * (DEMO_CELSIUS + 273.15) / F
    rows = {"cahi": 2, "capool": 2, "hhdemo": 3, "kcaf": 1, "pas": 0}
    order = ["cahi", "capool", "hhdemo", "kcaf", "pas"]
    S = {}
    r = 0
    for k in order:
        if k in on:
            S[k] = list(st[r:r + rows[k]])
            r += rows[k]
    cai = S["capool"][0] if ("capool" in on and not init) else 0.0

    def cnexp(x, xinf, tau):
        return x + (-math.expm1(-dt / tau)) * (xinf - x)

    def vtrap(x, y):
        return y * (1 - x / y / 2) if abs(x / y) < 1e-6 else x / math.expm1(x / y)

    # state phase
    if "cahi" in on:
        minf = 1 / (1 + math.exp(-(v + 20) / 6))
        mtau = 0.5 + 2 * math.exp(-((v + 20) / 25) ** 2)
        hinf = 1 / (1 + math.exp((v + 45) / 7))
        m, h = S["cahi"]
        S["cahi"] = [minf, hinf] if init else [cnexp(m, minf, mtau), cnexp(h, hinf, 80.0)]
    if "capool" in on:
        tau, shell, rest = prm["capool"]
        if init:
            cai = rest
        else:
            c, ica = S["capool"]
            b = -1.0 / tau
            a = -ica * 1e4 / (2 * F * shell) + rest / tau
            cai = c + (-math.expm1(b * dt)) * (-a / b - c)
        S["capool"][0] = cai
    if "hhdemo" in on:
        q = 3 ** ((DEMO_CELSIUS - 6.3) / 10)
        am, bm = 0.1 * vtrap(-(v + 40), 10), 4 * math.exp(-(v + 65) / 18)
        ah, bh = 0.07 * math.exp(-(v + 65) / 20), 1 / (math.exp(-(v + 35) / 10) + 1)
        an, bn = 0.01 * vtrap(-(v + 55), 10), 0.125 * math.exp(-(v + 65) / 80)
        inf = [am / (am + bm), ah / (ah + bh), an / (an + bn)]
        tau = [1 / (q * (am + bm)), 1 / (q * (ah + bh)), 1 / (q * (an + bn))]
        S["hhdemo"] = inf if init else [cnexp(x, i, t) for x, i, t in zip(S["hhdemo"], inf, tau)]
    if "kcaf" in on:
        gbar, kd, tauz = prm["kcaf"]
        c = cai if cai >= 1e-9 else 1e-9
        zinf = c * c / (c * c + kd * kd)
        S["kcaf"] = [zinf] if init else [cnexp(S["kcaf"][0], zinf, tauz)]
    # current phase
    eca = ktf / 2 * math.log(2.0 / cai) if cai > 0 else math.inf
    I = G = ica_tot = 0.0
    if "cahi" in on:
        m, h = S["cahi"]
        g = prm["cahi"][0] * m * m * h
        ica = g * (v - eca)
        I += ica
        G += g
        ica_tot += ica
    if "hhdemo" in on:
        m, h, n = S["hhdemo"]
        gna, gk = prm["hhdemo"][0] * m ** 3 * h, prm["hhdemo"][1] * n ** 4
        I += gna * (v - DEMO_REV["na"]) + gk * (v - DEMO_REV["k"])
        G += gna + gk
    if "kcaf" in on:
        g = prm["kcaf"][0] * S["kcaf"][0]
        I += g * (v - DEMO_REV["k"])
        G += g
    if "pas" in on:
        I += prm["pas"][0] * (v - prm["pas"][1])
        G += prm["pas"][0]
    if "capool" in on:
        S["capool"][1] = ica_tot
    out = [x for k in order if k in on for x in S[k]]
    return np.array(out), I, G


def test_demo_layout():
    g = _demo()
    assert g.mechs == ("cahi", "capool", "hhdemo", "kcaf", "pas")
    assert g.params == ("gbar_cahi", "tau_capool", "shell_capool", "cai_rest_capool", "gnabar_hhdemo",
                        "gkbar_hhdemo", "gbar_kcaf", "kd_kcaf", "tauz_kcaf", "g_pas", "e_pas")
    assert g.state_rows == (2, 2, 3, 1, 0)   # capool: cai and the carried total ica
    assert g.param_defaults[g.param_index("gnabar_hhdemo")] == 0.12


@pytest.mark.parametrize("init", [True, False])
def test_demo_matches_numpy(tmp_path, init):
    g = _demo()
    L = _host_lib(g, tmp_path / "demo")
    rng = np.random.default_rng(3)
    sets = [["pas"], ["hhdemo"], ["capool"], ["cahi", "capool"], ["capool", "kcaf"],
            ["cahi", "capool", "hhdemo", "kcaf", "pas"]]
    for on in sets:
        for v in np.concatenate([np.linspace(-100, 40, 15), [-40.0, -55.0, -65.0, -20.0]]):
            rows = sum(g.state_rows[g.mech_index(k)] for k in on)
            st = np.zeros((max(rows, 1), 32))
            st[:, 0] = rng.uniform(0.05, 0.95, max(rows, 1))
            r = 0
            for k in g.mechs:
                if k in on:
                    if k == "capool":
                        st[r, 0] = rng.uniform(1e-5, 2e-3)
                        st[r + 1, 0] = rng.uniform(-0.01, 0.0)
                    r += g.state_rows[g.mech_index(k)]
            prm = {"cahi": [0.002], "capool": [40.0, 0.3, 2e-4], "hhdemo": [0.12, 0.036], "kcaf": [0.003, 4e-4, 8.0],
                   "pas": [3e-4, -68.0]}
            pvals = [x for k in g.mechs if k in on for x in prm[k]]
            pr = np.zeros((max(len(pvals), 1), 32), dtype=np.float32)
            pr[:len(pvals), 0] = pvals
            prm32 = {k: [float(np.float32(x)) for x in vals] for k, vals in prm.items()}
            mask = sum(1 << g.mech_index(k) for k in on)
            s_gen, I_gen, G_gen = _run_gen(L, init, mask, float(v), 0.025, st, pr)
            s_np, I_np, G_np = _demo_numpy(on, init, float(v), 0.025, st[:rows, 0], prm32)
            np.testing.assert_allclose(s_gen[:rows], s_np, rtol=1e-9, atol=1e-15, err_msg=f"{on} v={v}")
            assert I_gen == pytest.approx(I_np, rel=1e-9, abs=1e-14), (on, v)
            assert G_gen == pytest.approx(G_np, rel=1e-9, abs=1e-14), (on, v)


def test_parameter_reads_name_their_index():
    """Every parameter the generated code reads goes through pload<R, P>
    with P the parameter's index in the set (the index a folded constant is
    looked up by): generator and kernel agree on what each constant is."""
    import re
    g = _demo()
    k_of = {f"m{k}_": m for k, m in enumerate(g.mechs)}
    found = 0
    for line in g.source.splitlines():
        m = re.search(r"(m\d+_)(\w+) = pload<R, (\d+)>\(pr, q \+ (\d+)\)", line)
        if not m:
            continue
        found += 1
        mech = k_of[m.group(1)]
        assert g.params[int(m.group(3))] == f"{m.group(2)}_{mech}", line
        assert int(m.group(3)) in g.mech_params[g.mech_index(mech)]
    assert found == g.n_params


def test_symbolic_linear_form_and_derivative():
    from neurogpu_b200 import nmodl
    p = nmodl.Parser(nmodl.tokenize("-ica*(10000)/(2*F*d) + (r - c)/t\n"))
    f = p.expr()
    a, b = nmodl.linear_form(f, "c")
    assert nmodl.free_vars(b) == {"t"}
    assert "c" not in nmodl.free_vars(a)
    e = nmodl.Parser(nmodl.tokenize("g*m*m*(v - e) + k*exp(v/2)\n")).expr()
    d = nmodl.simplify(nmodl.diff(e, "v"))
    env = {"v": 1.3, "g": 2.0, "m": 0.5, "e": -3.0, "k": 0.25}

    def ev(x):
        return eval(_py(x), {"exp": math.exp, "log": math.log}, env)
    h = 1e-6
    num = (ev(nmodl.subst(e, "v", nmodl.Num(1.3 + h))) - ev(nmodl.subst(e, "v", nmodl.Num(1.3 - h)))) / (2 * h)
    assert ev(d) == pytest.approx(num, rel=1e-7)


def _py(x):
    from neurogpu_b200 import nmodl
    if isinstance(x, nmodl.Num):
        return repr(x.v)
    if isinstance(x, nmodl.Var):
        return x.name
    if isinstance(x, nmodl.Un):
        return f"(-{_py(x.e)})"
    if isinstance(x, nmodl.Call):
        return f"{x.name}({', '.join(_py(a) for a in x.args)})"
    op = "**" if x.op == "^" else x.op
    return f"({_py(x.l)} {op} {_py(x.r)})"


@pytest.mark.parametrize("text,msg", [
    ("NEURON { SUFFIX k1 }\nSTATE { a }\nNET_RECEIVE (w) { a = a + w }\n", "NET_RECEIVE"),
    ("NEURON { SUFFIX q }\nSTATE { x }\nBREAKPOINT { SOLVE d METHOD cnexp }\nDERIVATIVE d { x' = -x*x }\n",
     "not linear"),
    ("NEURON { SUFFIX q }\nSTATE { x }\nBREAKPOINT { SOLVE d METHOD runge }\nDERIVATIVE d { x' = -x }\n",
     "not supported"),
    ("NEURON { SUFFIX q NONSPECIFIC_CURRENT i }\nASSIGNED { i }\nBREAKPOINT { i = gx*v }\n", "unknown name"),
])
def test_unsupported_input_is_an_error(text, msg):
    from neurogpu_b200 import nmodl
    with pytest.raises(nmodl.NmodlError, match=msg):
        nmodl.generate({"q": text})


def _compare_with_handwritten(gen, ms, msid, deps, hp, L, special):
    import sys
    sys.path.insert(0, str(ROOT / "tests"))
    from test_channels_host import PROBE_LIB, PROBE_SRC
    if not PROBE_LIB.exists():
        subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
                        str(PROBE_SRC), "-o", str(PROBE_LIB)], check=True, capture_output=True)
    H = C.CDLL(str(PROBE_LIB))
    H.probe_node_f64.restype = None
    rng = np.random.default_rng(1)
    n = ms.n_mech
    worst = 0.0
    for trial in range(900):
        on = sorted(set([trial % n] + deps.get(trial % n, []))) if trial < 700 else \
            sorted(set(rng.choice(n, rng.integers(1, n), replace=False).tolist()))
        mask = sum(1 << k for k in on)
        nst = sum(gen.state_rows[k] for k in on)
        npr = sum(len(hp[k]) for k in on)
        st = np.zeros((max(nst, 1), 32))
        st[:, 0] = rng.uniform(0, 1, max(nst, 1))
        r = 0
        for k in on:
            if k == special:
                st[r, 0] = rng.uniform(5e-5, 5e-3)
                st[r + 1, 0] = rng.uniform(-0.02, 0)
            r += gen.state_rows[k]
        pr = np.zeros((max(npr, 1), 32), dtype=np.float32)
        pr[:, 0] = np.abs(rng.normal(0.5, 0.3, max(npr, 1))) + 0.05
        v = float(rng.choice([rng.uniform(-110, 50), -27.0, -38.0, -66.0, -32.0, -60.0, -154.9, -17.0, -64.4, -35.0]))
        for init in (0, 1):
            s1 = st.copy()
            I1, G1 = C.c_double(), C.c_double()
            H.probe_node_f64(msid, init, mask, C.c_double(v), C.c_double(0.025), s1.ctypes.data, pr.ctypes.data,
                             C.byref(I1), C.byref(G1))
            s2, I2, G2 = _run_gen(L, init, mask, v, 0.025, st, pr)
            for a, b in [(I1.value, I2), (G1.value, G2)] + list(zip(s1[:nst, 0], s2[:nst])):
                worst = max(worst, abs(a - b) / max(abs(a), abs(b), 1e-30))
    return worst


@pytest.mark.skipif(not TTPC_MODS.exists(), reason="the reference's .mod files are not present")
def test_generated_ttpc_matches_handwritten(tmp_path):
    from neurogpu_b200 import nmodl
    from neurogpu_b200.mechsets import TTPC
    gen = nmodl.generate_from_files(sorted(p for p in TTPC_MODS.glob("*.mod") if p.stem != "branching"),
                                    celsius=34.0, reversal={"na": 50.0, "k": -85.0})
    assert gen.mechs == TTPC.mechs and gen.params == TTPC.params and gen.mech_params == TTPC.mech_params
    L = _host_lib(gen, tmp_path / "ttpc")
    worst = _compare_with_handwritten(gen, TTPC, 0, {0: [2], 1: [2], 11: [2]}, [list(x) for x in TTPC.mech_params],
                                      L, special=2)
    print(f"generated TTPC vs hand-written: max relative difference {worst:.2e}")
    assert worst < 1e-9


@pytest.mark.skipif(not MAINEN_MODS.exists(), reason="the reference's .mod files are not present")
def test_generated_mainen_matches_handwritten(tmp_path):
    from neurogpu_b200 import nmodl
    from neurogpu_b200.mechsets import MAINEN
    gen = nmodl.generate_from_files(sorted(p for p in MAINEN_MODS.glob("*.mod") if p.stem != "branching"),
                                    celsius=37.0, reversal={"na": 60.0, "k": -90.0}, constants=MAINEN_CONSTANTS)
    assert gen.mechs == MAINEN.mechs
    hp = [list(x) for x in MAINEN.mech_params]
    hp[0] = [0]  # the hand-written ca reads gbar only (cao is a constant)
    L = _host_lib(gen, tmp_path / "mainen")
    worst = _compare_with_handwritten(gen, MAINEN, 1, {0: [1, 2], 2: [1]}, hp, L, special=1)
    print(f"generated Mainen vs hand-written: max relative difference {worst:.2e}")
    assert worst < 1e-9


@pytest.mark.parametrize("precision", [0, 1])
def test_defined_set_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch, precision):
    from neurogpu_b200 import _ffi
    g = _demo().register()
    assert g.id >= 2
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    masks = np.array([0b11111, 0b00100], dtype=np.uint32)
    rc = L.ngpu_jit_build(g.id, precision, masks.ctypes.data, len(masks), 10, 0, C.byref(n))
    assert rc == 0, L.ngpu_last_error()
    assert n.value > 0
    nm, npar = C.c_int32(), C.c_int32()
    assert L.ngpu_mechset_info(g.id, C.byref(nm), C.byref(npar)) == 0
    assert (nm.value, npar.value) == (g.n_mech, g.n_params)


# ------------------------------------------------------------------- GPU
def _demo_workload(g, n_sets=8, t_stop=60.0, dt=0.025, seed=9):
    from neurogpu_b200 import configs
    from neurogpu_b200.model import build_model
    rng = np.random.default_rng(seed)
    secs = configs.hh_morphology(rng, 120)
    mechs = {"soma": ("cahi", "capool", "hhdemo", "kcaf", "pas"), "dend": ("cahi", "capool", "kcaf", "pas"),
             "axon": ("hhdemo", "pas")}
    cell = build_model(secs, g, ("soma", "dend", "axon"), mechs, ra=100.0,
                       cm_of_region={"soma": 1.0, "dend": 1.0, "axon": 1.0})
    base = np.array(g.param_defaults, dtype=np.float64)
    base[g.param_index("g_pas")] = 3e-4
    base[g.param_index("e_pas")] = -65.0
    mult = np.exp(rng.uniform(np.log(0.7), np.log(1.4), (n_sets, 1)))
    params = np.broadcast_to(base[None, :, None], (n_sets, g.n_params, cell.n_sections)).copy()
    params[:, g.param_index("gnabar_hhdemo"), :] *= mult
    nt = int(round(t_stop / dt))
    amps = configs.step_amps([0.3, 0.8], nt, dt, 5.0, 50.0)
    return configs.Workload("demo", cell, params.astype(np.float32), amps, dt, 0, float(cell.area[0]),
                            np.array([0], dtype=np.int32), -65.0)


def _sim(w, precision):
    from neurogpu_b200.sim import Simulator
    sim = Simulator(w.cell, w.n_sets, w.n_stim, precision)
    sim.set_params(w.params)
    sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    sim.set_recording(w.rec_nodes)
    sim.init(w.v_init)
    sim.advance(0, w.nt)
    out, bad = sim.trace(), sim.n_bad()
    sim.close()
    return out, bad


@pytest.mark.gpu
def test_defined_set_runs_fp32_against_fp64(ngpu_built):
    g = _demo().register()
    w = _demo_workload(g)
    v32, bad32 = _sim(w, "fp32")
    v64, bad64 = _sim(w, "fp64")
    assert bad32 == 0 and bad64 == 0
    n_spk = int(sum(((v64[..., :-1] < -20) & (v64[..., 1:] >= -20)).sum() for _ in [0]))
    err, mism = spike_time_error(v32, v64, w.dt)
    sub = subthreshold_error(v32, v64, w.dt)
    print(f"demo set: {n_spk} spikes; FP32 vs FP64 spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert n_spk > 0
    assert mism == 0 and err <= 0.05 and sub <= 0.1


@pytest.mark.gpu
def test_defined_set_folded_matches_loaded(ngpu_built, monkeypatch):
    """The demo set with its uniform parameters compiled in against the same
    set reading every parameter, FP32: a constant under the wrong index would
    change the traces by far more than the bounds."""
    g = _demo().register()
    w = _demo_workload(g)
    monkeypatch.setenv("NGPU_PARAM_FOLD", "1")
    from neurogpu_b200.sim import Simulator
    probe = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
    probe.set_params(w.params)
    probe.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    probe.set_recording(w.rec_nodes)
    probe.init(w.v_init)
    assert probe.param_folds() >= 5
    probe.close()
    a, bad_a = _sim(w, "fp32")
    monkeypatch.setenv("NGPU_PARAM_FOLD", "0")
    b, bad_b = _sim(w, "fp32")
    assert bad_a == 0 and bad_b == 0
    err, mism = spike_time_error(a, b, w.dt)
    sub = subthreshold_error(a, b, w.dt)
    print(f"demo set folded vs loaded: spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert mism == 0 and err <= 0.05 and sub <= 0.01


@pytest.mark.gpu
def test_defined_set_batch_matches_separate_runs(ngpu_built, monkeypatch):
    """Two demo-set simulations of different trees in one batch (one
    runtime-compiled kernel for both, with the parameters both hold at one
    value compiled in) against each run alone reading every parameter."""
    from neurogpu_b200.sim import Batch, Simulator
    g = _demo().register()
    ws = [_demo_workload(g, seed=9), _demo_workload(g, seed=10)]

    def sims():
        out = []
        for w in ws:
            s = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
            s.set_params(w.params)
            s.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
            s.set_recording(w.rec_nodes)
            out.append(s)
        return out
    monkeypatch.setenv("NGPU_PARAM_FOLD", "0")
    ref = []
    for s, w in zip(sims(), ws):
        s.init(w.v_init)
        s.advance(0, w.nt)
        ref.append(s.trace())
        s.close()
    monkeypatch.setenv("NGPU_PARAM_FOLD", "1")
    ss = sims()
    b = Batch(ss)
    assert ss[0].param_folds() >= 5
    b.init(ws[0].v_init)
    b.advance(0, ws[0].nt)
    for s, r, w in zip(ss, ref, ws):
        got = s.trace()
        assert s.n_bad() == 0
        err, mism = spike_time_error(got, r, w.dt)
        sub = subthreshold_error(got, r, w.dt)
        assert mism == 0 and err <= 0.05 and sub <= 0.01, (err, sub)
    b.close()
    for s in ss:
        s.close()


@pytest.mark.gpu
def test_generated_pas_matches_builtin(ngpu_built):
    """A set generated from nothing but NEURON's pas, on the passive cable
    workload, against the built-in TTPC set's pas."""
    from dataclasses import replace

    from neurogpu_b200 import configs, nmodl
    w = configs.passive_cable(n_sets=16, t_stop=60.0)
    g = nmodl.generate({}, name="pas_only", celsius=34.0).register()
    assert g.mechs == ("pas",)
    cell = replace(w.cell, mechset=g, mech_mask=np.ones((1, w.cell.n_nodes), dtype=np.uint8))
    params = np.zeros((w.n_sets, 2, cell.n_sections), dtype=np.float32)
    from neurogpu_b200.mechsets import TTPC
    params[:, 0] = w.params[:, TTPC.param_index("g_pas")]
    params[:, 1] = w.params[:, TTPC.param_index("e_pas")]
    wg = replace(w, cell=cell, params=params)
    a, bad_a = _sim(w, "fp32")
    b, bad_b = _sim(wg, "fp32")
    assert bad_a == 0 and bad_b == 0
    d = float(np.max(np.abs(a.astype(np.float64) - b)))
    print(f"generated pas vs built-in pas: max |dV| {d:.2e} mV")
    assert d <= 1e-3
