"""Uneven batches: several morphologies (200 / 800 / 1500 / 3000 compartments,
HH-type channels) in one launch, the whole run as one CUDA graph, the warp
autotuner, and the FP32 batch against the FP64 oracle on a sample."""
import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error

pytestmark = pytest.mark.gpu

SIZES = (200, 800, 1500, 3000)


@pytest.fixture(scope="module")
def workloads():
    from neurogpu_b200 import configs
    # 80 ms: the protocols step on at 50 ms, so the sample spikes
    return configs.uneven_batch(n_sets=4 * 40, sizes=SIZES, t_stop=80.0, levels=(0.2, 0.6, 1.0))


def _sims(workloads, warps=(0, 0, 0, 0), precision="fp32"):
    from neurogpu_b200.sim import Simulator
    sims = []
    for w, W in zip(workloads, warps):
        s = Simulator(w.cell, w.n_sets, w.n_stim, precision, n_warps=W)
        s.set_params(w.params)
        s.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        s.set_recording(np.array([0, w.cell.n_nodes // 2], dtype=np.int32))
        sims.append(s)
    return sims


def test_batch_equals_separate_launches(ngpu_built, workloads, monkeypatch):
    """One launch over four morphologies with different warp counts gives
    bitwise the traces of four separate launches.  A batch folds only the
    parameters its members share, a single launch every uniform one, so both
    sides run without folding here (folded batches: the tests below)."""
    from neurogpu_b200.sim import Batch
    warps = (2, 4, 6, 8)
    ref = []
    monkeypatch.setenv("NGPU_PARAM_FOLD", "0")
    sims0 = _sims(workloads, warps)
    for s, w in zip(sims0, workloads):
        s.init(w.v_init)
        s.advance(0, 300)
        s.advance(300, w.nt - 300)
        ref.append(s.trace())
        s.close()
    sims = _sims(workloads, warps)
    b = Batch(sims)
    b.init(workloads[0].v_init)
    b.advance(0, 300)
    b.advance(300, workloads[0].nt - 300)
    for s, r in zip(sims, ref):
        got = s.trace()
        assert np.all(np.isfinite(got))
        assert np.array_equal(got, r)
        assert s.n_bad() == 0
    b.close()


def _batch_run(workloads, fold, monkeypatch, change=None):
    from neurogpu_b200.sim import Batch
    monkeypatch.setenv("NGPU_PARAM_FOLD", "1" if fold else "0")
    sims = _sims(workloads)
    b = Batch(sims)
    if change is not None:  # new values for member 1 after the batch exists
        sims[1].set_params(change)
    n_folds = sims[0].param_folds()
    b.init(workloads[0].v_init)
    b.advance(0, workloads[0].nt)
    out = [s.trace() for s in sims]
    assert all(s.n_bad() == 0 for s in sims)
    b.close()
    for s in sims:
        s.close()
    return out, n_folds


def _close(a, b, dt):
    for x, y in zip(a, b):
        err, mism = spike_time_error(x, y, dt)
        sub = subthreshold_error(x, y, dt)
        assert mism == 0 and err <= 0.05 and sub <= 0.01, (err, sub)


def test_batch_folds_the_parameters_its_members_share(ngpu_built, workloads, monkeypatch):
    """The batch's kernel compiles in the parameters that hold one value in
    every member (the HH kinetic constants): within the FP32 parity bounds of
    the batch that loads them."""
    folded, n = _batch_run(workloads, True, monkeypatch)
    loaded, n0 = _batch_run(workloads, False, monkeypatch)
    assert n >= 15 and n0 == 0
    _close(folded, loaded, float(workloads[0].dt))


def test_member_with_new_values_refolds_the_batch(ngpu_built, workloads, monkeypatch):
    """A member given new values after the batch exists (e_pas made to vary
    by set) breaks one of the batch's folds: the batch's kernel is rebuilt
    without it, and the run matches the unfolded batch on the same values
    (a kernel that kept the old constant would miss by millivolts)."""
    w = workloads[1]
    p2 = w.params.copy()
    p2[:, w.cell.mechset.param_index("e_pas"), :] += np.linspace(-3.0, 3.0, w.n_sets, dtype=np.float32)[:, None]
    folded, n = _batch_run(workloads, True, monkeypatch, change=p2)
    loaded, _ = _batch_run(workloads, False, monkeypatch, change=p2)
    base, n_base = _batch_run(workloads, True, monkeypatch)
    assert n == n_base - 1
    _close(folded, loaded, float(w.dt))


def test_graph_run_equals_batch(ngpu_built, workloads):
    import torch
    from neurogpu_b200.sim import Batch
    sims = _sims(workloads)
    b = Batch(sims)
    b.init(workloads[0].v_init)
    b.advance(0, workloads[0].nt)
    ref = [s.trace() for s in sims]
    stream = torch.cuda.Stream()
    for _ in range(2):                       # second call replays the captured graph
        b.run_graph(workloads[0].v_init, workloads[0].nt, 128, stream)
        stream.synchronize()
        for s, r in zip(sims, ref):
            assert np.array_equal(s.trace(), r)
    b.close()


def test_autotuner_picks_a_candidate(ngpu_built, workloads):
    from neurogpu_b200 import autotune
    w = workloads[2]
    res = autotune.tune_warps(w.cell, w.params, w.amps, w.dts, w.stim_node, w.stim_area, w.rec_nodes, w.v_init,
                              candidates=(2, 4, 8), steps=100, warmup=20, items=(2, 3))
    assert res["n_warps"] in (2, 4, 8) and res["items_per_warp"] in (2, 3) and len(res["ms_per_step"]) == 6
    assert autotune.tune_warps(w.cell, w.params, w.amps, w.dts, w.stim_node, w.stim_area, w.rec_nodes,
                               w.v_init, candidates=(2, 4, 8), items=(2, 3)) is res      # cached


def test_uneven_batch_fp64_vs_oracle_sample(ngpu_built, oracle, workloads):
    """An FP64 batch (its runtime-specialised kernel, shared parameters
    compiled in) against the FP64 oracle on a sample: 2 sets x every
    protocol of each morphology, max |dV| <= 1e-5 mV (the float32 output's
    rounding)."""
    from neurogpu_b200.sim import Batch
    sims = _sims(workloads, precision="fp64")
    # members this small default to CTAs of more than 8 warps; the batch
    # kernel takes up to 8, so joining the batch splits them again
    assert max(s.layout()["cta_warps"] for s in sims) > 8
    b = Batch(sims)
    assert all(s.layout()["cta_warps"] <= 8 for s in sims)
    assert sims[0].param_folds() >= 15
    b.init(workloads[0].v_init)
    b.advance(0, workloads[0].nt)
    for s, w in zip(sims, workloads):
        got = s.trace()[:2, :, :1].astype(np.float64)
        ref = oracle.run_workload(w.subset(n_sets=2))
        err = float(np.max(np.abs(got - ref)))
        print(f"{w.name}: FP64 batch max|dV| {err:.2e} mV")
        assert err <= 1e-5
    b.close()


def test_uneven_batch_fp32_vs_oracle_sample(ngpu_built, oracle, workloads):
    """FP32 batch vs the FP64 oracle on a sample: 2 sets x every protocol of
    each morphology (spike time <= 0.05 ms, <= 0.1 mV away from spikes)."""
    from neurogpu_b200.sim import Batch
    sims = _sims(workloads)
    b = Batch(sims)
    b.init(workloads[0].v_init)
    b.advance(0, workloads[0].nt)
    for s, w in zip(sims, workloads):
        got = s.trace()[:2, :, :1].astype(np.float64)
        ref = oracle.run_workload(w.subset(n_sets=2))
        st, mism = spike_time_error(got, ref, w.dt)
        sub = subthreshold_error(got, ref, w.dt)
        print(f"{w.name}: spike {st:.4f} ms, mismatches {mism}, away from spikes {sub:.4f} mV")
        assert mism == 0 and st <= 0.05 and sub <= 0.1
    b.close()
