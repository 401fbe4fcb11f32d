"""The reference-facing driver surface: AllParams mapping, eFEL-named
features and their score combination (efel_ext.py), the multi-stimulus
evaluator, and the neuroGPU-compatible command line."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error
from neurogpu_b200 import evaluator as ev
from neurogpu_b200 import formats

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"
CLI = ROOT / "neurogpu_b200" / "bin" / "neuroGPU"


def test_allparams_from_mapping(tmp_path):
    tmpl = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    ind = [0, 12300, 0, 12301, 12300, 0]
    rows = ev.allparams_from_mapping([[10.5, 20.25], [30.0, 4e-5]], tmpl, ind, {5: 9.0},
                                     out_path=tmp_path / "AllParams.csv")
    np.testing.assert_array_equal(rows, [[1, 10.5, 3, 20.25, 10.5, 9], [1, 30, 3, 4e-5, 30, 9]])
    back = formats.read_params_csv(tmp_path / "AllParams.csv", 3, 2, True)   # 2 params x 3 sections
    np.testing.assert_allclose(back.reshape(2, -1), rows.astype(np.float32), rtol=1e-6)
    assert (tmp_path / "AllParams.csv").read_text().splitlines()[0] == "2"


def _two_spikes(dt=0.1):
    t = np.cumsum(np.full(6000, dt))
    v = np.full(t.size, -70.0)
    v[t > 400] = -65.0
    for tp in (150.0, 250.0):                     # triangles: 1 ms up to +30, 2 ms down to -75
        up = (t > tp - 1.0) & (t <= tp)
        v[up] = -70.0 + 100.0 * (t[up] - (tp - 1.0))
        dn = (t > tp) & (t <= tp + 2.0)
        v[dn] = 30.0 - 52.5 * (t[dn] - tp)
    return t, v


def test_efel_features_known_answers():
    t, v = _two_spikes()
    f = ev.efel_features(t, v)
    assert f["voltage_base"][0] == pytest.approx(-70.0)
    np.testing.assert_allclose(f["peak_time"], [150.0, 250.0], atol=0.11)
    np.testing.assert_allclose(f["AP_amplitude"], [100.0, 100.0], atol=1.0)
    np.testing.assert_allclose(f["AHP_depth"], [-5.0, -5.0], atol=0.6)
    np.testing.assert_allclose(f["spike_half_width"], [1.5, 1.5], atol=0.11)
    assert f["voltage_after_stim"][0] == pytest.approx(-65.0)
    flat = ev.efel_features(t, np.full(t.size, -70.0))
    assert flat["peak_time"] is None and flat["AP_amplitude"] is None


def test_efel_eval_penalties_and_zeros():
    t, v = _two_spikes()
    bad = v.copy()
    bad[10] = np.nan
    flat = np.full(t.size, -70.0)
    res = ev.efel_eval([v], np.stack([v, bad, flat]), t)
    np.testing.assert_array_equal(res[0], np.zeros(7))
    np.testing.assert_array_equal(res[1], np.full(7, 100000.0))
    assert res[2][ev.ALL_FEATURES.index("AP_amplitude")] == 1000      # missing feature
    assert res[2][ev.ALL_FEATURES.index("chi")] == pytest.approx(np.mean(np.abs(v - flat)))


def test_evaluator_with_fake_simulator():
    m = formats.read_data_dir(GOLD / "ttpc512", stim_index=0, params_file="AllParams_reference.csv")
    tmpl = m.raw["file_params"][0].reshape(-1).astype(np.float64)
    ind = np.zeros_like(tmpl)
    ind[[0, 5]] = [12300, 12301]
    t, v = _two_spikes()
    nt = 6000
    stims = np.zeros((2, nt), dtype=np.float32)
    m.dts = np.full(nt, 0.1, dtype=np.float32)

    def fake_run(cell, params, amps, dts, stim_node, area, rec, v_init):
        out = np.empty((params.shape[0], amps.shape[0], 1, amps.shape[1]), dtype=np.float32)
        for k in range(params.shape[0]):                    # individual k: trace shifted by k mV
            out[k, :, 0, :] = v + k
        return out

    e = ev.MultiStimEvaluator(m, stims, np.stack([v, v]), np.zeros(2), np.ones(2), (tmpl, ind, {}),
                              run=fake_run)
    scores = e.evaluate_with_lists([[0.1, 0.2], [0.3, 0.4]])
    assert len(scores) == 2 and scores[0].shape == (14,) and len(e.objectives) == 14
    np.testing.assert_allclose(scores[0], np.zeros(14), atol=1e-6)    # float32 traces
    assert scores[1][ev.ALL_FEATURES.index("voltage_base")] == pytest.approx(1.0)


def _data_dir(tmp_path, n_sets):
    sys.path.insert(0, str(GOLD))
    import make_ref_traces as M
    params = M.param_sets(n_sets, 0.2)
    M.write_run_dir(tmp_path, params)
    return tmp_path, params


def test_cli_check(tmp_path):
    root, _ = _data_dir(tmp_path, 4)
    p = subprocess.run([sys.executable, str(CLI), "--check"], cwd=root / "bin", capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert "512 nodes, 4 sets, 1 stimuli x 3168 steps" in p.stdout
    (root / "Data" / "Sim.csv").unlink()
    p = subprocess.run([sys.executable, str(CLI), "--check"], cwd=root / "bin", capture_output=True, text=True)
    assert p.returncode == 1 and "cannot read" in p.stderr


@pytest.mark.gpu
def test_cli_matches_reference_gpu(ngpu_built, tmp_path):
    """neuroGPU run in the reference's directory layout on the 16 parameter
    sets of the committed reference traces: VHotP0.dat and RunTimes.csv in
    the reference's formats, traces within the parity bounds of the
    reference's own GPU output."""
    root, params = _data_dir(tmp_path, 16)
    p = subprocess.run([sys.executable, str(CLI)], cwd=root / "bin", capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    v = formats.read_vhot(root / "Data" / "VHotP0.dat").reshape(16, 3168)
    n, ms = (root / "Data" / "RunTimes.csv").read_text().strip().split(",")
    assert int(n) == 16 and float(ms) > 0
    z = np.load(GOLD / "ref_ttpc512_traces.npz")
    assert np.array_equal(z["params"].view(np.uint32), params.view(np.uint32))
    ref = z["traces"].astype(np.float64)
    st, mism = spike_time_error(v, ref, 0.1)
    assert mism == 0 and st <= 0.05
    assert subthreshold_error(v, ref, 0.1) <= 0.2   # the reference itself is 0.095 mV from the FP64 oracle
