"""Integration methods of DERIVATIVE blocks besides cnexp in the NMODL
generator (neurogpu_b200/nmodl.py): derivimplicit (implicit Euler; for an
equation linear in its state one exact step, x' = (x + dt a) / (1 - dt b))
and euler (explicit: every derivative at the states the step started from,
then the updates).

Demo mechanisms (tests/golden/mod_methods, written for these tests): a
calcium pool by derivimplicit and a two-state channel by euler whose second
state relaxes towards the first.  The generated code, compiled for the host
in FP64, is checked against numpy statements of the two methods; NVRTC
builds it for sm_100a; coupled derivimplicit systems and nonlinear
equations are errors."""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

from test_nmodl import _host_lib, _run_gen

DIR = Path(__file__).resolve().parent / "golden" / "mod_methods"
REV = {"k": -77.0}
F = 96485.309


def _gen():
    from neurogpu_b200 import nmodl
    return nmodl.generate_from_files(sorted(DIR.glob("*.mod")), name="methods", celsius=6.3, reversal=REV)


def _cabe(init, dt, cai0, ica, taur, cainf, depth):
    if init:
        return cainf
    a = -ica * 1e4 / (2 * F * depth) + cainf / taur
    b = -1.0 / taur
    return (cai0 + dt * a) / (1.0 - dt * b)


def _keul(init, v, dt, m0, h0):
    minf = 1.0 / (1.0 + math.exp(-(v + 30.0) / 8.0))
    mtau = 2.0 + 3.0 * math.exp(-((v + 40.0) / 20.0) ** 2)
    if init:
        return minf, minf
    dm, dh = (minf - m0) / mtau, (m0 - h0) / 20.0
    return m0 + dt * dm, h0 + dt * dh


@pytest.mark.parametrize("init", [True, False])
def test_methods_match_numpy(tmp_path, init):
    g = _gen()
    assert g.mechs == ("cabe", "keul", "pas") and g.state_rows == (2, 2, 0)
    L = _host_lib(g, tmp_path / "methods")
    rng = np.random.default_rng(4)
    taur, cainf, depth, gbar = (float(np.float32(x)) for x in (80.0, 1e-4, 0.5, 0.01))
    for v in np.linspace(-90.0, 30.0, 13):
        for dt in (0.025, 0.5, 5.0):
            st = np.zeros((4, 32))
            st[0, 0] = rng.uniform(5e-5, 2e-3)        # cai
            st[1, 0] = rng.uniform(-0.02, 0.0)        # the carried total ica
            st[2, 0], st[3, 0] = rng.uniform(0.0, 1.0, 2)
            pr = np.zeros((4, 32), dtype=np.float32)
            pr[:4, 0] = [taur, cainf, depth, gbar]
            s_gen, I_gen, G_gen = _run_gen(L, init, 0b011, float(v), dt, st, pr)
            cai = _cabe(init, dt, st[0, 0], st[1, 0], taur, cainf, depth)
            m, h = _keul(init, float(v), dt, st[2, 0], st[3, 0])
            assert s_gen[0] == pytest.approx(cai, rel=1e-12), (v, dt)
            assert s_gen[2] == pytest.approx(m, rel=1e-12, abs=1e-15) and s_gen[3] == pytest.approx(h, rel=1e-12, abs=1e-15)
            gk = gbar * m * h
            assert I_gen == pytest.approx(gk * (v - REV["k"]), rel=1e-12, abs=1e-15)
            assert G_gen == pytest.approx(gk, rel=1e-12, abs=1e-15)


def test_derivimplicit_is_unconditionally_stable(tmp_path):
    """A step far longer than the pool's time constant lands between the
    state and its fixed point (implicit Euler), never beyond it."""
    g = _gen()
    L = _host_lib(g, tmp_path / "methods")
    st = np.zeros((4, 32))
    st[0, 0] = 5e-3
    pr = np.zeros((4, 32), dtype=np.float32)
    pr[:4, 0] = [80.0, 1e-4, 0.5, 0.0]
    s, _, _ = _run_gen(L, False, 0b001, -65.0, 1e4, st, pr)
    assert float(np.float32(1e-4)) < s[0] < 5e-3


@pytest.mark.parametrize("text,msg", [
    ("NEURON { SUFFIX q }\nSTATE { x y }\nBREAKPOINT { SOLVE d METHOD derivimplicit }\n"
     "DERIVATIVE d { x' = y - x  y' = -y }\n", "coupled"),
    ("NEURON { SUFFIX q }\nSTATE { x }\nBREAKPOINT { SOLVE d METHOD derivimplicit }\n"
     "DERIVATIVE d { x' = -x*x }\n", "linear in their state"),
])
def test_method_errors(text, msg):
    from neurogpu_b200 import nmodl
    with pytest.raises(nmodl.NmodlError, match=msg):
        nmodl.generate({"q": text})


def test_method_set_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch):
    from neurogpu_b200 import _ffi
    g = _gen().register()
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    masks = np.array([0b111, 0b110], dtype=np.uint32)
    assert L.ngpu_jit_build(g.id, 0, masks.ctypes.data, len(masks), 10, 0, C.byref(n)) == 0, L.ngpu_last_error()
    assert n.value > 0
