"""The autotuner: recording cadence from a pilot trace (CPU), layout and
shape selection by timing (GPU)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def pilot(oracle):
    """FP64 oracle traces of the HH-type cell, recorded every step (dt 0.025 ms)."""
    from neurogpu_b200 import configs
    w = configs.hh_active(n_sets=4, t_stop=120.0)
    return oracle.run_workload(w)[:, :, 0, :], w.dt


def test_every_step_loses_nothing(pilot):
    from neurogpu_b200.autotune import cadence_errors
    v, _ = pilot
    e = cadence_errors(v, 1)
    assert e == {"count_mismatches": 0, "spike_shift_steps": 0.0, "peak_drop_mV": 0.0}


def test_cadence_meets_its_tolerances(pilot):
    from neurogpu_b200.autotune import cadence_errors, tune_cadence
    v, dt = pilot
    n_spikes = int(((v[..., :-1] < -20) & (v[..., 1:] >= -20)).sum())
    assert n_spikes > 20
    r = tune_cadence(v, dt, spike_tol_ms=0.05, peak_tol_mv=1.0)
    k = r["rec_every"]
    e = cadence_errors(v, k)
    assert e["count_mismatches"] == 0 and e["spike_shift_steps"] * dt <= 0.05 and e["peak_drop_mV"] <= 1.0
    # the next coarser candidate breaks a tolerance (the search stops there)
    coarser = [c for c in r["errors"] if c > k]
    assert coarser, r
    c = coarser[0]
    ec = r["errors"][c]
    assert ec["count_mismatches"] > 0 or ec["spike_shift_steps"] * dt > 0.05 or ec["peak_drop_mV"] > 1.0
    # looser tolerances never give a finer cadence
    assert tune_cadence(v, dt, spike_tol_ms=0.2, peak_tol_mv=5.0)["rec_every"] >= k


def test_subthreshold_trace_takes_the_coarsest_cadence():
    from neurogpu_b200.autotune import tune_cadence
    t = np.arange(4000) * 0.025
    v = -70.0 + 5.0 * np.sin(t / 20.0)
    assert tune_cadence(v[None, :], 0.025)["rec_every"] == 40


@pytest.mark.gpu
def test_tune_times_both_layouts_on_a_small_batch(ngpu_built):
    from neurogpu_b200 import autotune, configs
    from neurogpu_b200.sim import Simulator
    w = configs.hh_active(n_sets=8, t_stop=5.0)
    r = autotune.tune(w.cell, w.params, w.amps, w.dts, w.stim_node, w.stim_area, w.rec_nodes, w.v_init,
                      steps=60, warmup=10, lane_shapes=((4, 2), (8, 3)), warp_shapes=((1, 32), (2, 16)))
    assert set(r["ms_per_step"]) == {"lane:4:2", "lane:8:3", "warp:1:32", "warp:2:16"}
    assert all(v > 0 for v in r["ms_per_step"].values())
    best = min(r["ms_per_step"], key=r["ms_per_step"].get)
    assert best == f"{r['layout']}:{r['n_warps']}:{r['items_per_warp']}"
    s = Simulator(w.cell, w.n_sets, w.n_stim, "fp32", n_warps=r["n_warps"], items_per_warp=r["items_per_warp"],
                  layout=r["layout"])
    assert s.layout() == {"layout": r["layout"], "cta_warps": r["n_warps"], "items": r["items_per_warp"]}
    s.close()
