"""Batched trace features (neurogpu_b200.features) on traces with known answers."""
import numpy as np
import pytest
import torch

from neurogpu_b200 import features as F


def _train(spike_times, dt=0.1, T=500.0, base=-70.0, ss=-65.0):
    t = np.arange(int(T / dt)) * dt
    v = np.full(t.size, base)
    v[(t >= 50) & (t < 450)] = ss
    for ts in spike_times:                       # 1 ms up to +30, 1 ms down to -75
        up = (t >= ts - 1.0) & (t < ts)
        v[up] = -70.0 + 100.0 * (t[up] - (ts - 1.0))
        dn = (t >= ts) & (t < ts + 1.0)
        v[dn] = 30.0 - 105.0 * (t[dn] - ts)
    return v


def test_spiking_and_silent_traces():
    dt = 0.1
    v = torch.tensor(np.stack([_train([100.0, 150.0, 220.0], dt), _train([], dt)]), dtype=torch.float32)
    f = F.extract(v, dt, 50.0, 450.0).numpy()
    k = {n: i for i, n in enumerate(F.FEATURES)}
    a, s = f[0], f[1]
    assert a[k["spike_count"]] == 3 and s[k["spike_count"]] == 0
    assert a[k["first_spike_latency"]] == pytest.approx(100.0 - 50.0 - 0.5, abs=0.25)
    assert a[k["mean_isi"]] == pytest.approx(60.0, abs=0.25)
    assert a[k["first_isi"]] == pytest.approx(50.0, abs=0.25) and a[k["last_isi"]] == pytest.approx(70.0, abs=0.25)
    assert a[k["adaptation"]] == pytest.approx(1.4, abs=0.02)
    assert a[k["ap_peak_mean"]] == pytest.approx(30.0, abs=1.0)
    assert a[k["voltage_base"]] == pytest.approx(-70.0) and a[k["steady_state"]] == pytest.approx(-65.0)
    assert s[k["first_spike_latency"]] == pytest.approx(400.0) and s[k["mean_isi"]] == pytest.approx(400.0)
    assert s[k["adaptation"]] == 1.0 and s[k["isi_cv"]] == 0.0
    assert np.all(np.isfinite(f))


def _compare(a, b, dt):
    """The CUDA kernel against the torch statement, feature by feature."""
    k = {n: i for i, n in enumerate(F.FEATURES)}
    a, b = a.cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(a[:, k["spike_count"]], b[:, k["spike_count"]])
    for name in ("first_spike_latency", "first_isi", "last_isi", "last_spike_time", "v_max", "v_min_stim"):
        np.testing.assert_allclose(a[:, k[name]], b[:, k[name]], rtol=1e-6, atol=1e-5, err_msg=name)
    for name in ("mean_isi", "isi_cv", "adaptation", "ap_peak_mean", "ap_peak_std", "ahp_mean", "ap_amplitude_mean",
                 "voltage_base", "steady_state", "voltage_after_stim", "v_mean_stim", "v_std_stim"):
        np.testing.assert_allclose(a[:, k[name]], b[:, k[name]], rtol=2e-5, atol=2e-4, err_msg=name)
    # time above half amplitude: the half level is rounded once in each statement, which can move
    # one sample across it per spike
    n = np.maximum(a[:, k["spike_count"]], 1)
    assert np.all(np.abs(a[:, k["time_above_half"]] - b[:, k["time_above_half"]]) <= dt / n + 1e-6)


@pytest.mark.gpu
def test_cuda_kernel_matches_torch_on_known_traces(ngpu_built):
    dt = 0.1
    trains = [[100.0, 150.0, 220.0], [], [60.0], [51.0, 449.5], list(np.arange(60.0, 440.0, 7.3)), [300.0, 301.5]]
    v = torch.tensor(np.stack([_train(s, dt) for s in trains]), dtype=torch.float32).cuda()
    _compare(F.extract_device(v, dt, 50.0, 450.0), F.extract(v, dt, 50.0, 450.0), dt)
    # a transposed (sample-major) view reads the same traces through the strides
    vt = v.t().contiguous().t()
    _compare(F.extract_device(vt, dt, 50.0, 450.0), F.extract(v, dt, 50.0, 450.0), dt)


@pytest.mark.gpu
def test_features_from_the_simulation_buffer(ngpu_built):
    """ngpu_sim_features reads the simulator's [sample][site][instance] buffer
    in place; the same features as the torch statement on the copied trace."""
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Simulator
    w = configs.hh_active(n_sets=64, t_stop=200.0, levels=(0.2, 0.5, 1.0))
    sim = Simulator(w.cell, w.n_sets, w.n_stim, "fp32")
    sim.set_params(w.params)
    sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    sim.set_recording(w.rec_nodes, 4)
    sim.init(w.v_init)
    sim.advance(0, w.nt)
    dts = w.dt * 4
    got = sim.features(dts, 50.0, 180.0)
    tr = torch.tensor(sim.trace()[:, :, 0, :]).cuda().reshape(w.n_sets * w.n_stim, -1)
    want = F.extract(tr, dts, 50.0, 180.0)
    sim.close()
    assert float(want[:, 0].sum()) > 0      # the batch spikes
    _compare(got.reshape(-1, F.N_FEATURES), want, dts)
