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

Config 3 is the exception, and the fixtures show why: the TTPC-like cell's
spike times are sensitive at the level of float32 rounding itself.  The FP64
oracle with every parameter nudged by one part in 1e7 (about one float32
ulp) moves its spikes by ~0.08 ms and its voltage by ~0.3 mV at 2000 ms
(the fixture's sens_* values), and the oracle's own float32 build (correctly
rounded libm, no GPU intrinsics) drifts by ~0.13 ms and ~1.1 mV (f32_*).  No
float32 arithmetic can follow this model within 0.05 ms over 2000 ms.  So
for config 3 the FP32 run of the whole batch must meet the strict bounds
over its first 250 ms and, over the full 2000 ms, stay within 1.5 x the
oracle's float32 build's deviation; and the FP64 kernel (precision "fp64",
here on the warp-instance layout) meets the strict bounds over the full
2000 ms.

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


def compare(name, got_full, dt, rows=None, horizon_ms=None):
    """got_full [n, n_stim, nt] GPU soma traces of the sampled sets (rows:
    their indices into the fixture's sets; default all, in order).  Spikes
    after horizon_ms are left out.  Returns the error summary."""
    fx, stride = _fixture(name)
    v_ref, spk, off = fx["v"], fx["spk"], fx["spk_off"]
    n, ns, nt = got_full.shape
    rows = np.arange(n) if rows is None else np.asarray(rows)
    if horizon_ms is not None:
        nt = min(nt, int(round(horizon_ms / dt)))
        got_full = got_full[..., :nt]
    assert v_ref.shape[1] == ns and rows.size == n
    win = int(round(WINDOW_MS / dt))
    worst_v, worst_t, mism, n_spk = 0.0, 0.0, 0, 0
    for jj, tr in enumerate(got_full.reshape(n * ns, nt)):
        j = rows[jj // ns] * ns + jj % ns   # the trace's index in the fixture
        s_ref = spk[off[j]:off[j + 1]]
        s_got = spike_times(tr, dt)
        if horizon_ms is not None:  # spikes within 1 ms of the cut are left out on both sides
            cut = (nt - 1) * dt - 1.0
            s_ref, s_got = s_ref[s_ref < cut], s_got[s_got < cut]
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
        b = v_ref.reshape(-1, v_ref.shape[-1])[j, :a.size].astype(np.float64)
        if keep.any():
            worst_v = max(worst_v, float(np.max(np.abs(a[keep] - b[keep]))))
    return {"traces": n * ns, "spikes": n_spk, "max_dv_away_mV": worst_v, "spike_err_ms": worst_t,
            "count_mismatches": mism}


def _check(name, res, tol_spike=TOL_SPIKE_MS, tol_mv=TOL_FP32_MV):
    print(f"\n{name}: {res}")
    assert res["count_mismatches"] == 0, res
    assert res["spike_err_ms"] <= tol_spike, res
    assert res["max_dv_away_mV"] <= tol_mv, res


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
def test_config2_full_batch_full_duration(ngpu_built):
    (w, sets, _), = _workloads()["hh_500ms"]
    sim = _setup(w)
    got = _sim_sampled(sim, w, sets, 8000)
    sim.close()
    _check("hh_500ms", compare("hh_500ms", got, w.dt))


@pytest.mark.gpu
def test_config3_full_batch_fp32(ngpu_built):
    """The whole TTPC-like batch, FP32 + Kahan, 2000 ms: strict bounds over
    the first 250 ms; over the full run, within 1.5 x the deviation of the
    oracle's own float32 build (see the module docstring)."""
    name = "ttpc_2000ms"
    (w, sets, _), = _workloads()[name]
    fx, _ = _fixture(name)
    sim = _setup(w)
    got = _sim_sampled(sim, w, sets, 8000)
    sim.close()
    for h in (250, 500, 1000, 1500):
        print(f"\n{name} FP32 first {h} ms: {compare(name, got, w.dt, horizon_ms=h)}")
    _check(name + " FP32 first 250 ms", compare(name, got, w.dt, horizon_ms=250))
    print(f"\n{name}: FP64 oracle under a {float(fx['sens_eps']):g} parameter nudge: spikes "
          f"{float(fx['sens_spike_ms']):.4f} ms, {float(fx['sens_dv_away_mV']):.4f} mV away from spikes; "
          f"the oracle's float32 build: {float(fx['f32_spike_ms']):.4f} ms, {float(fx['f32_dv_away_mV']):.4f} mV")
    _check(name + " FP32 2000 ms", compare(name, got, w.dt), tol_spike=1.5 * float(fx["f32_spike_ms"]),
           tol_mv=1.5 * float(fx["f32_dv_away_mV"]))


@pytest.mark.gpu
def test_config3_fp64_full_duration(ngpu_built):
    """Two of the sampled sets (6 instances), FP64 kernel on the
    warp-instance layout, 2000 ms: the strict bounds."""
    from neurogpu_b200.sim import Simulator
    name = "ttpc_2000ms"
    (w, sets, _), = _workloads()[name]
    ws = w.take(sets[:2])
    sim = Simulator(ws.cell, ws.n_sets, ws.n_stim, "fp64", layout="warp")
    sim.set_params(ws.params)
    sim.set_stimulus(ws.amps, ws.dts, ws.stim_node, ws.stim_area)
    sim.set_recording(ws.rec_nodes)
    got = _sim_sampled(sim, ws, np.arange(2), 8000)
    sim.close()
    _check(name + " FP64", compare(name, got, w.dt, rows=[0, 1]))


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
