"""The reference's own shipped model: the 512-node BBP TTPC cell of
GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/Data (tests/golden/ttpc512), read with
the reference-format readers, 3168 steps of 0.1 ms, 16 parameter sets (the
shipped set and seeded +-20 % scalings of it, as
tests/golden/make_ref_traces.py makes them).

The model joins near zero-area compartments (couplings ~3e21) to ordinary
ones (~1e-1 .. 1e11), which an FP32 solve survives only in the kernel's
excess form.

  * FP64 kernel vs FP64 oracle: max |dV| <= 1e-5 mV.
  * FP32 kernel vs FP64 oracle: spike-time error <= 0.05 ms, no spike-count
    mismatch, max |dV| <= 0.1 mV away from spikes (outside +-2 ms).
  * tests/golden/ref_ttpc512_traces.npz (the reference's GPU simulator on the
    same inputs, when committed): the oracle and the FP32 kernel against it
    with the same spike-time bound; away from spikes both against the
    reference's own FP32 deviation from the oracle plus 0.1 mV.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))

TOL_FP64_MV = 1e-5
TOL_FP32_MV = 0.1
TOL_SPIKE_MS = 0.05
N_SETS = 16
REF_TRACES = GOLD / "ref_ttpc512_traces.npz"


@pytest.fixture(scope="module")
def shipped():
    import make_ref_traces as M
    m = M.model_inputs()
    params = M.param_sets(N_SETS, 0.2)
    if REF_TRACES.exists():
        z = np.load(REF_TRACES)
        assert np.array_equal(z["params"].view(np.uint32), params.view(np.uint32))
    return m, params


@pytest.fixture(scope="module")
def oracle_f64(oracle, shipped):
    m, params = shipped
    c = m.cell
    return oracle.run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask, params,
                      m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init)


def _gpu(shipped, precision):
    from neurogpu_b200.sim import run
    m, params = shipped
    return run(m.cell, params, m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init,
               precision=precision).astype(np.float64)


def test_oracle_f32_floor(oracle, shipped, oracle_f64):
    """How far FP32 channel arithmetic alone (with an FP64 solve) drifts on
    this model: the floor any FP32 simulator shares."""
    m, params = shipped
    c = m.cell
    f32 = oracle.run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask, params,
                     m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init, precision="f32")
    st, mism = spike_time_error(f32, oracle_f64, 0.1)
    sub = subthreshold_error(f32, oracle_f64, 0.1)
    print(f"oracle f32 vs f64: spike {st:.4f} ms, mismatches {mism}, away from spikes {sub:.4f} mV")
    assert mism == 0 and st <= TOL_SPIKE_MS


@pytest.mark.gpu
def test_fp64_kernel_matches_oracle(ngpu_built, shipped, oracle_f64):
    got = _gpu(shipped, "fp64")
    err = np.max(np.abs(got - oracle_f64))
    assert err <= TOL_FP64_MV, f"FP64 max|dV| = {err:.3e} mV"


@pytest.mark.gpu
def test_fp32_kernel_matches_oracle(ngpu_built, shipped, oracle_f64):
    got = _gpu(shipped, "fp32")
    assert np.all(np.isfinite(got))
    st, mism = spike_time_error(got, oracle_f64, 0.1)
    sub = subthreshold_error(got, oracle_f64, 0.1)
    print(f"FP32 kernel vs oracle: spike {st:.4f} ms, mismatches {mism}, away from spikes {sub:.4f} mV, "
          f"max {np.max(np.abs(got - oracle_f64)):.3f} mV")
    assert mism == 0
    assert st <= TOL_SPIKE_MS
    assert sub <= TOL_FP32_MV


def _ref_traces():
    if not REF_TRACES.exists():
        pytest.skip("reference traces not generated (tests/golden/make_ref_traces.py --save)")
    return np.load(REF_TRACES)["traces"].astype(np.float64)[:, None, None, :]


def test_reference_gpu_traces_match_oracle(shipped, oracle_f64):
    ref = _ref_traces()
    st, mism = spike_time_error(oracle_f64, ref, 0.1)
    sub = subthreshold_error(oracle_f64, ref, 0.1)
    print(f"oracle f64 vs reference GPU: spike {st:.4f} ms, mismatches {mism}, away from spikes {sub:.4f} mV")
    assert mism == 0 and st <= TOL_SPIKE_MS


@pytest.mark.gpu
def test_fp32_kernel_matches_reference_gpu(ngpu_built, shipped, oracle_f64):
    ref = _ref_traces()
    got = _gpu(shipped, "fp32")
    st, mism = spike_time_error(got, ref, 0.1)
    sub = subthreshold_error(got, ref, 0.1)
    ref_sub = subthreshold_error(oracle_f64, ref, 0.1)
    print(f"FP32 kernel vs reference GPU: spike {st:.4f} ms, mismatches {mism}, away from spikes {sub:.4f} mV "
          f"(reference vs oracle {ref_sub:.4f} mV)")
    assert mism == 0 and st <= TOL_SPIKE_MS
    assert sub <= ref_sub + TOL_FP32_MV
