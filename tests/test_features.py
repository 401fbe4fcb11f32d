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
