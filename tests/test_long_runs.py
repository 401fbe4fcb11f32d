"""Parity at the benchmark configurations' stated durations.

The GPU runs the whole batch of a configuration, FP32 with the
Kahan-compensated voltage, for its full duration; a sample of its parameter
sets is compared with the FP64 oracle (fixtures made by
tests/golden/make_long_runs.py from oracle/oracle.c, which restates the
reference's step, GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/CudaStuff.cu:
227-330):

  config 2  HH-type 500 compartments, 1024 sets x 3 protocols, 500 ms
            (20,000 steps); 16 sets
  config 3  TTPC-like 1501 compartments, 4096 sets x 3 protocols, 2000 ms
            (80,000 steps); 8 sets
  config 4  uneven batch, 8192 sets over 200/800/1500/3000-compartment trees
            x 5 protocols, 500 ms, one CUDA graph; a 1 % sample (82 sets)

Bounds (the targets of the FP32 simulator): spike-time error <= 0.05 ms over
matched spikes, no trace with a different spike count, and max |dV| <= 0.1 mV
at the 1 ms samples farther than 2 ms from any spike of either trace.

The CPU test pins the fixtures to the oracle: a fresh oracle run of the first
50 ms of a sampled set reproduces the stored samples exactly.
"""
import functools

import numpy as np
import pytest

from helpers import spike_times

TOL_SPIKE_MS = 0.05
TOL_FP32_MV = 0.1
WINDOW_MS = 2.0

GOLDEN = None


def _golden():
    global GOLDEN
    if GOLDEN is None:
        from pathlib import Path
        GOLDEN = dict(np.load(Path(__file__).resolve().parent / "golden" / "long_runs.npz"))
    return GOLDEN


def _fixture(name):
    g = _golden()
    return {k.split("/", 1)[1]: v for k, v in g.items() if k.startswith(name + "/")}, int(g["stride"])


@functools.cache
def _workloads():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_long_runs
    return make_long_runs.workloads()


def compare(name, got_full, dt):
    """got_full [n, n_stim, nt] GPU soma traces of the sampled sets, in the
    fixture's order.  Returns the error summary."""
    fx, stride = _fixture(name)
    v_ref, spk, off = fx["v"], fx["spk"], fx["spk_off"]
    n, ns, nt = got_full.shape
    assert v_ref.shape[:2] == (n, ns)
    win = int(round(WINDOW_MS / dt))
    worst_v, worst_t, mism, n_spk = 0.0, 0.0, 0, 0
    for j, tr in enumerate(got_full.reshape(n * ns, nt)):
        s_ref = spk[off[j]:off[j + 1]]
        s_got = spike_times(tr, dt)
        n_spk += s_ref.size
        if s_got.size != s_ref.size:
            mism += 1
        elif s_ref.size:
            worst_t = max(worst_t, float(np.max(np.abs(s_got - s_ref))))
        keep = np.ones(nt, dtype=bool)
        for t in np.concatenate([s_ref, s_got]):
            k = int(t / dt)
            keep[max(0, k - win):k + win + 1] = False
        keep = keep[::stride]
        a = tr[::stride].astype(np.float64)
        b = v_ref.reshape(n * ns, -1)[j].astype(np.float64)
        if keep.any():
            worst_v = max(worst_v, float(np.max(np.abs(a[keep] - b[keep]))))
    return {"traces": n * ns, "spikes": n_spk, "max_dv_away_mV": worst_v, "spike_err_ms": worst_t,
            "count_mismatches": mism}


def _check(name, res):
    print(f"\n{name}: {res}")
    assert res["count_mismatches"] == 0, res
    assert res["spike_err_ms"] <= TOL_SPIKE_MS, res
    assert res["max_dv_away_mV"] <= TOL_FP32_MV, res


def _sim_sampled(sim, w, sets, chunk):
    """Advance a set-up simulation of workload w through its steps in
    launches of `chunk` and return the sampled sets' soma traces
    [len(sets), n_stim, nt]."""
    sim.init(w.v_init)
    t = 0
    while t < w.nt:
        c = min(chunk, w.nt - t)
        sim.advance(t, c)
        t += c
    assert sim.n_bad() == 0
    return _gather(sim, sets)


def _gather(sim, sets):
    import torch
    out = torch.empty((sim.n_sets, sim.n_stim, sim.n_rec, sim.n_samples), dtype=torch.float32, device="cuda")
    sim.trace_into(out.data_ptr())
    torch.cuda.synchronize()
    idx = torch.as_tensor(np.asarray(sets), device="cuda")
    got = out.index_select(0, idx)[:, :, 0, :].cpu().numpy()
    del out
    torch.cuda.empty_cache()
    return got


def _setup(w, **shape):
    from neurogpu_b200.sim import Simulator
    sim = Simulator(w.cell, w.n_sets, w.n_stim, "fp32", **shape)
    sim.set_params(w.params)
    sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    sim.set_recording(w.rec_nodes)
    return sim


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["hh_500ms", "ttpc_2000ms"])
def test_full_batch_full_duration(ngpu_built, name):
    (w, sets, _), = _workloads()[name]
    sim = _setup(w)
    got = _sim_sampled(sim, w, sets, 8000)
    sim.close()
    _check(name, compare(name, got, w.dt))


@pytest.mark.gpu
def test_uneven_batch_one_graph(ngpu_built):
    """Config 4: the four trees as one batch, init and every chunk of the
    500 ms run captured as one CUDA graph and replayed once."""
    import torch
    from neurogpu_b200.sim import Batch
    parts = _workloads()["uneven_500ms"]
    sims = [_setup(w) for w, _, _ in parts]
    batch = Batch(sims)
    stream = torch.cuda.Stream()
    nt = parts[0][0].nt
    batch.run_graph(parts[0][0].v_init, nt, 2000, stream)
    stream.synchronize()
    got = []
    for (w, sets, _), s in zip(parts, sims):
        assert s.n_bad() == 0
        got.append(_gather(s, sets))
    batch.close()
    for s in sims:
        s.close()
    _check("uneven_500ms", compare("uneven_500ms", np.concatenate(got), parts[0][0].dt))


@pytest.mark.parametrize("name", ["hh_500ms", "ttpc_2000ms", "uneven_500ms"])
def test_fixture_matches_oracle_prefix(oracle, name):
    """The stored samples of the first sampled set (every protocol) equal a
    fresh oracle run of its first 50 ms, sample for sample."""
    fx, stride = _fixture(name)
    w, sets, _ = _workloads()[name][0]
    ws = w.take(sets[:1]).subset(nt=2000)
    ref = oracle.run_workload(ws)[:, :, 0, ::stride].astype(np.float32)
    np.testing.assert_array_equal(ref[0], fx["v"][0, :, :ref.shape[-1]])
    assert fx["sets"][0] == sets[0]
