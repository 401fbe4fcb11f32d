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
    bitwise the traces of four separate launches.  A batch's kernel compiles
    no parameters in as constants, so the separate launches run without
    folding too."""
    from neurogpu_b200.sim import Batch
    warps = (2, 4, 6, 8)
    ref = []
    monkeypatch.setenv("NGPU_PARAM_FOLD", "0")
    sims0 = _sims(workloads, warps)
    monkeypatch.delenv("NGPU_PARAM_FOLD")
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
