"""CPU check of the product's channel equations against the oracle.

The product's channel headers (neurogpu_b200/csrc/channels_*.cuh) are
compiled for the host in FP64 (tests/native/chan_probe.cu) and compared, one
mechanism at a time, with the oracle's node functions, which restate the
reference's generated channel code.  Both sides are FP64, so the bound is
1e-9 relative (the product uses efun series / analytic conductance where the
oracle follows the reference's literal expressions)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PROBE_SRC = ROOT / "tests" / "native" / "chan_probe.cu"
PROBE_LIB = ROOT / "tests" / "native" / "libchanprobe.so"

# product state rows per mechanism -> oracle state index; "cai"/"ica" are the
# oracle's trailing per-node variables (n_states + 0 / + 2)
TTPC_ROWS = [[0, 1], [2, 3], ["cai", "ica"], [5], [6], [7, 8], [9, 10], [11, 12], [13, 14],
             [15, 16], [], [17], [18]]
MAINEN_ROWS = [[0, 1], [2, "ica"], [3], [4], [5], [6, 7], [], [], []]
TTPC_DEPS = {0: [2], 1: [2], 11: [2]}      # Ca currents / SK need CaDynamics
MAINEN_DEPS = {0: [1, 2], 2: [1]}          # ca needs cad (and kca, see configs); kca reads cad


@pytest.fixture(scope="module")
def probe():
    srcs = [PROBE_SRC] + list((ROOT / "neurogpu_b200" / "csrc").glob("channels_*.cuh")) + \
        [ROOT / "neurogpu_b200" / "csrc" / "ngpu_math.cuh"]
    if not PROBE_LIB.exists() or any(p.stat().st_mtime > PROBE_LIB.stat().st_mtime for p in srcs):
        subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
                        "--expt-relaxed-constexpr", str(PROBE_SRC), "-o", str(PROBE_LIB)],
                       check=True, capture_output=True)
    L = C.CDLL(str(PROBE_LIB))
    L.probe_node_f64.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_double, C.c_double, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def _nominal(mechset_name, rng):
    from neurogpu_b200 import configs
    from neurogpu_b200.mechsets import MAINEN, TTPC
    if mechset_name == "ttpc":
        ms = TTPC
        p = np.zeros(ms.n_params)
        for d in (configs.TTPC_FIXED, configs.TTPC_NOMINAL["axon"], configs.TTPC_NOMINAL["soma"]):
            for k, v in d.items():
                p[ms.param_index(k)] = v
        p[ms.param_index("gK_Pstbar_K_Pst")] = 0.97
        p[ms.param_index("gK_Tstbar_K_Tst")] = 0.09
        p[ms.param_index("gIhbar_Ih")] = 8e-5
        p[ms.param_index("gImbar_Im")] = 1.43e-4
    else:
        ms = MAINEN
        p = np.zeros(ms.n_params)
        for d in (configs.MAINEN_FIXED, configs.MAINEN_NOMINAL["soma"]):
            for k, v in d.items():
                p[ms.param_index(k)] = v
        p[ms.param_index("g_pas2")] = 1e-5
        p[ms.param_index("e_pas2")] = -60.0
        p[ms.param_index("g_pasx")] = 2e-5
        p[ms.param_index("e_pasx")] = -80.0
    scale = np.exp(rng.uniform(np.log(0.3), np.log(3.0), p.size))
    gates = np.array(["bar" in n or n.startswith("g_") for n in ms.params])
    p = np.where(gates, p * scale, p)
    return ms, p


def _compare(probe, oracle, mechset_name, mechs_on, v, dt, rng, init):
    ms, p = _nominal(mechset_name, rng)
    rows = TTPC_ROWS if mechset_name == "ttpc" else MAINEN_ROWS
    NS = {"ttpc": 19, "mainen": 8}[mechset_name]
    CAI, ECA, ICA = NS, NS + 1, NS + 2
    mask = 0
    mk = np.zeros(ms.n_mech, dtype=np.uint8)
    for k in mechs_on:
        mask |= 1 << k
        mk[k] = 1
    # product layout: compact state rows / parameter rows in mechanism order
    prow_params = [pi for k in mechs_on for pi in ms.mech_params[k]
                   if not (mechset_name == "mainen" and k == 0 and pi == 1)]
    srow_map = [r for k in mechs_on for r in rows[k]]
    ost = np.zeros(NS + 3)
    st = np.zeros((max(1, len(srow_map)), 32))
    for j, r in enumerate(srow_map):
        if r == "ica":
            val = rng.uniform(-0.02, 0.0)
        elif r == "cai":
            val = rng.uniform(5e-5, 5e-3)
        else:
            val = rng.uniform(0.0, 1.0)
        st[j, 0] = val
        ost[{"cai": CAI, "ica": ICA}.get(r, r) if isinstance(r, str) else r] = val
    if mechset_name == "mainen" and 1 in mechs_on:
        ost[CAI] = ost[2]
    if mechset_name == "ttpc" and 2 not in mechs_on:
        ost[CAI] = 0.0
    ktf = 1000. * 8.3134 * (ms.celsius + 273.15) / 96485.309
    ost[ECA] = ktf / 2 * np.log(2.0 / ost[CAI]) if ost[CAI] > 0 else 0.0
    pr = np.zeros((max(1, len(prow_params)), 32), dtype=np.float32)
    pr[:len(prow_params), 0] = p[prow_params]
    pf = p.astype(np.float32).astype(np.float64)  # the product reads float32 parameters
    I, G = C.c_double(), C.c_double()
    probe.probe_node_f64(ms.id, int(init), mask, v, dt, st.ctypes.data, pr.ctypes.data,
                         C.byref(I), C.byref(G))
    L = oracle.lib()
    mkp = mk.ctypes.data
    if init:
        ost[:] = 0.0
        L.ong_node_init_f64(ms.id, mkp, v, pf.ctypes.data, ost.ctypes.data)
    else:
        L.ong_node_deriv_f64(ms.id, mkp, dt, v, pf.ctypes.data, ost.ctypes.data)
    ost[ICA] = 0.0
    g = C.c_double()
    Io = L.ong_node_current_f64(ms.id, mkp, v, pf.ctypes.data, ost.ctypes.data, C.byref(g))
    for j, r in enumerate(srow_map):
        want = ost[{"cai": CAI, "ica": ICA}.get(r, r) if isinstance(r, str) else r]
        assert st[j, 0] == pytest.approx(want, rel=1e-9, abs=1e-15), (mechset_name, mechs_on, r, v)
    assert I.value == pytest.approx(Io, rel=1e-9, abs=1e-14), (mechset_name, mechs_on, v)
    assert G.value == pytest.approx(g.value, rel=1e-9, abs=1e-14), (mechset_name, mechs_on, v)


@pytest.mark.parametrize("mechset_name", ["ttpc", "mainen"])
@pytest.mark.parametrize("init", [True, False])
def test_each_mechanism_matches_oracle(probe, oracle, mechset_name, init):
    rng = np.random.default_rng(7)
    n_mech = 13 if mechset_name == "ttpc" else 9
    deps = TTPC_DEPS if mechset_name == "ttpc" else MAINEN_DEPS
    for k in range(n_mech):
        on = sorted(set([k] + deps.get(k, [])))
        for v in np.concatenate([np.linspace(-110, 50, 23), [-38.0, -27.0, -66.0, -35.0, -32.0, -60.0, -17.0, -64.4, -154.9]]):
            _compare(probe, oracle, mechset_name, on, float(v), 0.025, rng, init)


@pytest.mark.parametrize("mechset_name", ["ttpc", "mainen"])
def test_all_mechanisms_together(probe, oracle, mechset_name):
    rng = np.random.default_rng(11)
    n_mech = 13 if mechset_name == "ttpc" else 9
    for v in np.linspace(-90, 30, 13):
        for init in (True, False):
            _compare(probe, oracle, mechset_name, list(range(n_mech)), float(v), 0.1, rng, init)


EFUN_PROBE = r'''
#include "channels_ttpc.cuh"
extern "C" void probe_pair_f32(float z, float* pos, float* neg) { ngpu::efun_pair<float>(z, *pos, *neg); }
extern "C" void probe_pair_f64(double z, double* pos, double* neg) { ngpu::efun_pair<double>(z, *pos, *neg); }
'''


def test_efun_pair_against_two_efuns(tmp_path):
    """efun_pair (one exponential for efun(z) and efun(-z)), compiled for the
    host from the channel header, against z/(e^z - 1) in FP64 over |z| <= 100:
    through the series switch at 1e-2 and past FP32's overflow of e^z
    (z > 88.7), where efun(-z) -> z.  The FP64 bound is the series' own
    truncation, z^4/720 < 1.4e-11 for |z| < 1e-2 (efun uses the same series)."""
    (tmp_path / "p.cu").write_text(EFUN_PROBE)
    r = subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
                        "-I", str(ROOT / "neurogpu_b200" / "csrc"), str(tmp_path / "p.cu"), "-o",
                        str(tmp_path / "libp.so")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    L = C.CDLL(str(tmp_path / "libp.so"))
    L.probe_pair_f32.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.probe_pair_f64.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]

    def efun(z):   # z / (e^z - 1), from expm1 so that it is exact near 0
        return 1.0 if z == 0.0 else z / np.expm1(z)

    zs = np.concatenate([np.linspace(-100, 100, 2001), [-1e-2, -9.9e-3, 0.0, 9.9e-3, 1e-2, 79.9, 80.1, 88.5, 89.0, 95.0]])
    for fn, ctype, rel in ((L.probe_pair_f64, C.c_double, 2e-11), (L.probe_pair_f32, C.c_float, 1e-5)):
        for z in zs:
            z = float(ctype(z).value)
            p, n = ctype(), ctype()
            fn(z, C.byref(p), C.byref(n))
            assert np.isfinite(p.value) and np.isfinite(n.value), z
            assert p.value == pytest.approx(efun(z), rel=rel, abs=1e-30), z
            assert n.value == pytest.approx(efun(-z), rel=rel, abs=1e-30), z
