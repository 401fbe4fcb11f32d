"""The eFEL features the reference's evaluator asks for (P/efel_ext.py:13),
checked against their published definitions (as restated in
neurogpu_b200.evaluator.efel_features) on piecewise-linear traces whose
features follow by hand from those definitions.

A spike here rises from -70 mV at t0 to +30 mV at t0 + 1 ms (100 mV/ms),
falls to -80 mV at t0 + 3 ms (-55 mV/ms) and recovers to -70 mV at t0 + 10 ms.
On such a trace numpy's central differences are exact inside each segment,
so AP begin is the rise's first sample (dV/dt 50 mV/ms there >= 10), the peak
is +30 mV, the half level (30 + -70) / 2 = -20 mV is crossed at t0 + 0.5 ms on
the way up and at t0 + 1 + 50/55 ms on the way down, and the AHP minimum is
-80 mV.  Window: stim 100-400 ms, threshold -30 mV (efel_ext.py:5-13).
"""
import numpy as np
import pytest

from neurogpu_b200 import evaluator as E

T = np.arange(5001) / 10.0           # 0 .. 500 ms, 0.1 ms samples, exact grid
HALF_WIDTH = 0.5 + 50.0 / 55.0       # from the half-level crossings above


def trace(spikes=(), rest=-70.0, t=T):
    """V(t): rest, with the spike shape above at each t0 in spikes."""
    knots_t, knots_v = [t[0]], [rest]
    for t0 in sorted(spikes):
        knots_t += [t0, t0 + 1.0, t0 + 3.0, t0 + 10.0]
        knots_v += [rest, 30.0, -80.0, rest]
    knots_t.append(t[-1] + 20.0)
    knots_v.append(rest)
    return np.interp(t, knots_t, knots_v)


def test_no_spikes():
    v = trace()
    v[(T > 150) & (T < 350)] = -60.0     # a subthreshold response
    f = E.efel_features(T, v)
    assert f["voltage_base"][0] == pytest.approx(-70.0)
    assert f["voltage_after_stim"][0] == pytest.approx(-70.0)
    for k in ("peak_time", "AP_amplitude", "spike_half_width", "AHP_depth"):
        assert f[k] is None


def test_one_spike():
    f = E.efel_features(T, trace([200.0]))
    np.testing.assert_allclose(f["peak_time"], [201.0])
    np.testing.assert_allclose(f["AP_amplitude"], [100.0])
    np.testing.assert_allclose(f["spike_half_width"], [HALF_WIDTH], rtol=1e-12)
    np.testing.assert_allclose(f["AHP_depth"], [-10.0])      # min -80 after the peak, base -70
    assert f["voltage_base"][0] == pytest.approx(-70.0)


def test_two_spikes():
    v = trace([150.0, 250.0])
    f = E.efel_features(T, v)
    np.testing.assert_allclose(f["peak_time"], [151.0, 251.0])
    np.testing.assert_allclose(f["AP_amplitude"], [100.0, 100.0])
    np.testing.assert_allclose(f["spike_half_width"], [HALF_WIDTH, HALF_WIDTH], rtol=1e-12)
    np.testing.assert_allclose(f["AHP_depth"], [-10.0, -10.0])


def test_spikes_at_the_window_edges():
    """Peaks at 90.0 ms (before stim_start) and 410.5 ms (after stim_end)
    are left out.  The peak at 100.5 ms (its rise starts at 99.5 ms) is in,
    with its AP begin at the window's first sample, stim_start, where V =
    -20 mV and dV/dt = 100 mV/ms: amplitude 50 mV, half level 5 mV.  The
    peak at 399.8 ms is in, and its AHP is the minimum up to stim_end,
    V(400) = 30 - 55 x 0.2 = 19 mV."""
    v = trace([89.0, 99.5, 398.8, 409.5])
    f = E.efel_features(T, v)
    np.testing.assert_allclose(f["peak_time"], [100.5, 399.8])
    np.testing.assert_allclose(f["AP_amplitude"], [30.0 - (-20.0), 100.0])
    ahp = f["AHP_depth"] + f["voltage_base"][0]          # the minima themselves
    np.testing.assert_allclose(ahp, [-80.0, 19.0], atol=1e-9)
    rise = 100.0 + (5.0 - (-20.0)) / 100.0               # V = -20 at 100.0 ms, +100 mV/ms
    fall = 100.5 + (30.0 - 5.0) / 55.0
    np.testing.assert_allclose(f["spike_half_width"], [fall - rise, HALF_WIDTH], rtol=1e-9)


def test_trace_ending_inside_the_stimulus():
    """A trace that ends at 300 ms, on the rise of a spike: no samples after
    the stimulus (voltage_after_stim None); the cut spike's peak is the last
    sample, and its fall never reaches the half level, so it has no width."""
    t = T[T <= 300.0]
    v = trace([200.0, 299.5], t=t)
    f = E.efel_features(t, v)
    assert f["voltage_after_stim"] is None
    np.testing.assert_allclose(f["peak_time"], [201.0, 300.0])
    np.testing.assert_allclose(f["spike_half_width"], [HALF_WIDTH], rtol=1e-12)


def test_threshold_is_the_evaluators():
    """A spike peaking at -35 mV stays below efel_ext.py's -30 mV threshold."""
    v = trace()
    v[(T >= 200.0) & (T <= 201.0)] = -35.0
    assert E.efel_features(T, v)["peak_time"] is None
