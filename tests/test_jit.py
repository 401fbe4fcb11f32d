"""Runtime specialisation of the advance kernel (NVRTC, ngpu_jit.h).

CPU: the generated translation unit compiles for sm_100a through the C ABI
(ngpu_jit_build; NVRTC needs no device) for both mechanism sets, and the
compiled image is reused from the on-disk cache.
GPU: FP32 simulations run the specialised kernel (ngpu_sim_classes > 0) and
agree with the ahead-of-time kernel (NGPU_JIT=0, generic channel code): the
same arithmetic with the mechanism tests folded, so traces agree to FP32
rounding order (bound: the FP32 parity bounds of test_gpu_parity, and the
subthreshold difference far below them).
"""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error


def _masks(w):
    m = w.cell.mech_mask.astype(np.int64)
    return np.unique((m << np.arange(m.shape[0])[:, None]).sum(0)).astype(np.uint32)


@pytest.mark.parametrize("name", ["ttpc_like", "hh_active"])
def test_jit_builds_for_sm100a(ngpu_built, tmp_path, monkeypatch, name):
    from neurogpu_b200 import _ffi, configs
    w = getattr(configs, name)(n_sets=2, t_stop=1.0)
    masks = _masks(w)
    monkeypatch.setenv("NGPU_JIT_CACHE", str(tmp_path))
    L = _ffi.lib()
    n = C.c_int64(0)
    rc = L.ngpu_jit_build(w.cell.mechset.id, 0, masks.ctypes.data, len(masks), 10, 0, C.byref(n))
    assert rc == 0, L.ngpu_last_error()
    assert n.value > 0
    cached = list(tmp_path.glob("*.cubin"))
    assert len(cached) == 1 and cached[0].stat().st_size == n.value
    n2 = C.c_int64(0)
    assert L.ngpu_jit_build(w.cell.mechset.id, 0, masks.ctypes.data, len(masks), 10, 0, C.byref(n2)) == 0
    assert n2.value == n.value


def test_jit_build_rejects_bad_arguments(ngpu_built):
    from neurogpu_b200 import _ffi
    L = _ffi.lib()
    n = C.c_int64(0)
    m = np.array([1], dtype=np.uint32)
    assert L.ngpu_jit_build(7, 0, m.ctypes.data, 1, 10, 0, C.byref(n)) != 0
    many = np.arange(1, 18, dtype=np.uint32)
    assert L.ngpu_jit_build(0, 0, many.ctypes.data, len(many), 10, 0, C.byref(n)) != 0


def _run(w, jit: bool):
    from neurogpu_b200.sim import Simulator
    old = os.environ.get("NGPU_JIT")
    os.environ["NGPU_JIT"] = "1" if jit else "0"
    try:
        sim = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
        sim.set_params(w.params)
        sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        sim.set_recording(w.rec_nodes)
        sim.init(w.v_init)
        sim.advance(0, w.nt)
        out, classes, bad = sim.trace(), sim.classes(), sim.n_bad()
        sim.close()
    finally:
        if old is None:
            os.environ.pop("NGPU_JIT", None)
        else:
            os.environ["NGPU_JIT"] = old
    return out, classes, bad


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ttpc_like", "hh_active"])
def test_specialised_kernel_matches_generic(ngpu_built, name):
    from neurogpu_b200 import _ffi, configs
    w = getattr(configs, name)(n_sets=16, t_stop=150.0)
    jit, n_cls, bad_j = _run(w, True)
    gen, n_gen, bad_g = _run(w, False)
    assert n_cls == len(_masks(w)), _ffi.lib().ngpu_jit_log()
    assert n_gen == 0
    assert bad_j == 0 and bad_g == 0
    dt = float(w.dt)
    err, mismatched = spike_time_error(jit, gen, dt)
    sub = subthreshold_error(jit, gen, dt)
    print(f"{name}: specialised vs generic: spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert mismatched == 0
    assert err <= 0.05
    assert sub <= 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("name,min_folds", [("ttpc_like", 4), ("hh_active", 15)])
def test_folded_parameters_match_loaded(ngpu_built, monkeypatch, name, min_folds):
    """Parameters that hold one value in every set and section (the models'
    kinetic constants) are compiled in as constants; the traces match those
    of the kernel that loads them, within the FP32 parity bounds (a constant
    lets the compiler evaluate an expression once, in its own rounding)."""
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Simulator
    w = getattr(configs, name)(n_sets=16, t_stop=150.0)

    def run(fold):
        monkeypatch.setenv("NGPU_PARAM_FOLD", "1" if fold else "0")
        sim = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
        sim.set_params(w.params)
        sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        sim.set_recording(w.rec_nodes)
        sim.init(w.v_init)
        sim.advance(0, w.nt)
        out, n, bad = sim.trace(), sim.param_folds(), sim.n_bad()
        sim.close()
        return out, n, bad
    folded, n_f, bad_f = run(True)
    loaded, n_l, bad_l = run(False)
    assert n_f >= min_folds and n_l == 0
    assert bad_f == 0 and bad_l == 0
    err, mismatched = spike_time_error(folded, loaded, float(w.dt))
    sub = subthreshold_error(folded, loaded, float(w.dt))
    print(f"{name}: {n_f} parameters folded; spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert mismatched == 0 and err <= 0.05 and sub <= 0.01


@pytest.mark.gpu
def test_new_parameters_mid_run_reselect_the_kernel(ngpu_built, monkeypatch):
    """set_params in the middle of a run with values that change which
    parameters are uniform: e_pas, compiled in as one constant at first, is
    then given a different value per set.  The rest of the run uses the new
    values (a kernel that kept the old constant would miss by millivolts):
    it matches the same run with folding off within the FP32 parity bounds."""
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Simulator
    w = configs.hh_active(n_sets=8, t_stop=100.0)
    p2 = w.params.copy()
    p2[:, w.cell.mechset.param_index("e_pas"), :] += np.linspace(-3.0, 3.0, w.n_sets, dtype=np.float32)[:, None]
    k = w.nt // 2

    def run(fold):
        monkeypatch.setenv("NGPU_PARAM_FOLD", "1" if fold else "0")
        sim = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
        sim.set_params(w.params)
        sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        sim.set_recording(w.rec_nodes)
        sim.init(w.v_init)
        n0 = sim.param_folds()
        sim.advance(0, k)
        sim.set_params(p2)
        n1 = sim.param_folds()
        sim.advance(k, w.nt - k)
        out = sim.trace()
        assert sim.n_bad() == 0
        sim.close()
        return out, n0, n1
    a, n0, n1 = run(True)
    c, m0, m1 = run(False)
    assert n1 == n0 - 1 and n0 > 0 and m0 == m1 == 0
    err, mismatched = spike_time_error(a, c, float(w.dt))
    sub = subthreshold_error(a, c, float(w.dt))
    assert mismatched == 0 and err <= 0.05 and sub <= 0.01, (err, sub)


@pytest.mark.gpu
@pytest.mark.parametrize("name,precision,frac", [("ttpc_like", "fp32", 0.8), ("hh_active", "fp32", 0.1),
                                                 ("ttpc_like", "fp64", 0.8)])
def test_shared_parameter_blocks_are_bitwise_neutral(ngpu_built, monkeypatch, name, precision, frac):
    """Sections whose parameter values repeat another section's read that
    section's rows: fewer rows are touched (the HH cell's values are per
    region; the TTPC-like cell's Ih and calcium densities vary with
    distance, section by section) and the traces are bitwise those of every
    section reading its own rows."""
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Simulator
    w = getattr(configs, name)(n_sets=16, t_stop=60.0)

    def run(dedup):
        monkeypatch.setenv("NGPU_PARAM_DEDUP", "1" if dedup else "0")
        sim = Simulator(w.cell, w.n_sets, w.n_stim, precision)
        sim.set_params(w.params)
        sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        sim.set_recording(w.rec_nodes)
        sim.init(w.v_init)
        sim.advance(0, w.nt)
        out, rows = sim.trace(), sim.param_rows()
        assert sim.n_bad() == 0
        sim.close()
        return out, rows
    shared, (read_s, total) = run(True)
    own, (read_o, total_o) = run(False)
    print(f"{name} {precision}: parameter rows read {read_s} of {total}")
    assert read_o == total_o == total and read_s < frac * total
    assert np.array_equal(shared, own)


@pytest.mark.gpu
def test_more_combinations_than_classes_match_the_oracle(ngpu_built, oracle):
    """A cell whose sections carry random subsets of the TTPC mechanisms has
    more distinct combinations than the 16 compiled classes: the other nodes
    run the generic channel code inside the specialised kernel (which is then
    compiled with it).  FP32 against the FP64 oracle within the parity
    bounds."""
    from dataclasses import replace

    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Simulator
    w = configs.ttpc_like(n_sets=8, t_stop=80.0)
    ms = w.cell.mechset
    rng = np.random.default_rng(12)
    n_sec = w.cell.n_sections
    sec_mask = (rng.random((ms.n_mech, n_sec)) < 0.45).astype(np.uint8)
    sec_mask[ms.mech_index("pas")] = 1
    ca = [ms.mech_index("Ca_HVA"), ms.mech_index("Ca_LVAst")]
    sec_mask[ms.mech_index("CaDynamics_E2")] |= sec_mask[ca].max(axis=0)   # calcium currents need the pool
    mask = sec_mask[:, np.asarray(w.cell.section)]
    n_comb = len({tuple(c) for c in mask.T})
    assert n_comb > 16
    # the workload gives values only where a region has the mechanism (a calcium
    # pool's decay is 0 elsewhere): kinetic and pool constants take the soma's
    # values in every section
    params = w.params.copy()
    soma = int(w.cell.section[0])
    for k, name in enumerate(ms.params):
        if "bar" not in name:
            params[:, k, :] = params[:, k, soma:soma + 1]
    wc = replace(w, cell=replace(w.cell, mech_mask=np.ascontiguousarray(mask)), params=np.ascontiguousarray(params))
    ref = oracle.run_workload(wc)
    assert np.all(np.isfinite(ref))
    sim = Simulator(wc.cell, wc.n_sets, wc.n_stim, "fp32")
    sim.set_params(wc.params)
    sim.set_stimulus(wc.amps, wc.dts, wc.stim_node, wc.stim_area)
    sim.set_recording(wc.rec_nodes)
    sim.init(wc.v_init)
    sim.advance(0, wc.nt)
    got = sim.trace().astype(np.float64)
    assert sim.classes() == 16 and sim.n_bad() == 0
    sim.close()
    err, mism = spike_time_error(got, ref, float(wc.dt))
    sub = subthreshold_error(got, ref, float(wc.dt))
    print(f"{n_comb} mechanism combinations: spike times {err:.2e} ms, subthreshold {sub:.2e} mV")
    assert mism == 0 and err <= 0.05 and sub <= 0.1
