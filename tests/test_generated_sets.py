"""Mechanism sets generated from the reference's .mod files, run on the GPU
against the FP64 oracle.

The generator (neurogpu_b200/nmodl.py; the reference's porting path is
NeuroGPU_Base/scripts/pyscripts/extractModel.py:1705-1812) turns the
reference's TTPC and Mainen .mod files into channel code that the runtime
compiler builds into the simulation kernel.  tests/golden/generated_sets/
holds its output (tests/golden/make_generated_sets.py), so these tests run
where the reference tree is absent.  The oracle (oracle/oracle.c) states the
same channels from the reference's generated C (GUI/BBP_TTPC_EXAMPLE/
pyNeuroGPU_unix/src/AllModels.cu, Figures/FigureS4_mainen/CParsed/
AllModels.cu), pinned against those files compiled for the host.

Bounds, as for the built-in sets (tests/test_gpu_parity.py): FP64 kernel
vs FP64 oracle max |dV| <= 1e-5 mV; FP32 kernel: spike-time error <= 0.05
ms, no spike-count mismatch, max |dV| <= 0.1 mV away from spikes.
"""
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_generated_sets as MG  # noqa: E402

TOL_FP64_MV = 1e-5
TOL_FP32_MV = 0.1
TOL_SPIKE_MS = 0.05

_REGISTERED = {}


def _gen(which):
    if which not in _REGISTERED:
        _REGISTERED[which] = MG.load(which).register()
    return _REGISTERED[which]


def _workloads(which):
    """(built-in workload for the oracle, the same workload on the generated set)."""
    from neurogpu_b200 import configs
    from neurogpu_b200.mechsets import MAINEN, TTPC
    g = _gen(which)
    if which == "ttpc":
        w = configs.ttpc_like(n_sets=12, t_stop=200.0)
        assert g.params == TTPC.params and g.mechs == TTPC.mechs
        params = w.params
    else:
        w = configs.hh_active(n_sets=24, t_stop=150.0)
        assert g.mechs == MAINEN.mechs
        # the generated ca takes cao as a constant: the workload must hold that value
        cao = w.params[:, MAINEN.param_index("cao_ca"), :]
        assert np.all(cao == np.float32(MG.MAINEN_CONSTANTS["ca"]["cao"]))
        params = np.ascontiguousarray(np.stack([w.params[:, MAINEN.param_index(n), :] for n in g.params], axis=1))
    return w, replace(w, cell=replace(w.cell, mechset=g), params=params)


def _run(w, precision):
    from neurogpu_b200.sim import Simulator
    sim = Simulator(w.cell, w.n_sets, w.n_stim, precision)
    sim.set_params(w.params)
    sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    sim.set_recording(w.rec_nodes)
    sim.init(w.v_init)
    sim.advance(0, w.nt)
    out = sim.trace()
    assert sim.n_bad() == 0
    assert sim.classes() > 0  # the runtime-compiled kernel with the generated channel code
    sim.close()
    return out


@pytest.fixture(scope="module")
def refs(oracle):
    out = {}
    for which in ("ttpc", "mainen"):
        from neurogpu_b200 import configs
        w = configs.ttpc_like(n_sets=12, t_stop=200.0) if which == "ttpc" else configs.hh_active(n_sets=24,
                                                                                                 t_stop=150.0)
        out[which] = oracle.run_workload(w)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ttpc", "mainen"])
def test_generated_set_fp64_matches_oracle(ngpu_built, refs, which):
    _, wg = _workloads(which)
    got = _run(wg, "fp64")
    err = float(np.max(np.abs(got.astype(np.float64) - refs[which])))
    print(f"{which} generated, FP64 vs oracle: max|dV| = {err:.3e} mV")
    assert err <= TOL_FP64_MV


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ttpc", "mainen"])
def test_generated_set_fp32_matches_oracle(ngpu_built, refs, which):
    w, wg = _workloads(which)
    got = _run(wg, "fp32").astype(np.float64)
    ref = refs[which]
    sub = subthreshold_error(got, ref, w.dt)
    st, mism = spike_time_error(got, ref, w.dt)
    print(f"{which} generated, FP32 vs oracle: away from spikes {sub:.3e} mV, spike times {st:.3e} ms, "
          f"count mismatches {mism}")
    assert mism == 0 and st <= TOL_SPIKE_MS and sub <= TOL_FP32_MV


@pytest.mark.skipif(not MG.TTPC_MODS.exists(), reason="the reference's .mod files are not present")
@pytest.mark.parametrize("which", ["ttpc", "mainen"])
def test_stored_sets_are_the_generators_output(which):
    stored = (MG.OUT / f"{which}.json").read_text()
    assert MG.to_json(MG.generate(which)) == stored
