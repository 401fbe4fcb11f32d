"""Drop-in for the reference's GA evaluator around the simulator.

Mirrors Figures/Figure4_DEAP/neurogpu_multistim_evaluator_par.py (class
``neurogpu_multistim_evaluator``), NeuroGPU_Base/scripts/pyscripts/efel_ext.py
and the parameter mapping of NeuroGPU_Base/scripts/template/
extractModel_mappings.py, with one change of mechanism: every stimulus of a
generation runs in one libngpu call instead of one neuroGPU process per
stimulus plus VHotP files.

Feature extraction: the reference calls eFEL (a git-pinned third-party
dependency, GUI/requirements.txt:23, absent here).  ``efel_features`` restates
the six eFEL features efel_ext.py asks for from eFEL's documented
definitions; no reference test pins eFEL's outputs, so these are unpinned.
The combination into scores (feature-list RMS differences, chi, NaN
penalties) follows efel_ext.py:23-96 exactly.
"""
from __future__ import annotations

import csv
import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable, Sequence

import numpy as np

from . import formats

# efel_ext.py:5-13
STIM_START = 100.0
STIM_END = 400.0
THRESHOLD = -30.0
DERIVATIVE_THRESHOLD = 10.0      # eFEL default, mV/ms
ALL_FEATURES = ["voltage_base", "AP_amplitude", "voltage_after_stim", "peak_time", "spike_half_width",
                "AHP_depth", "chi"]
PARAM_INDICATOR_BASE = 12300.0   # extractModel_mappings.py:271


def nrnMread(fileName) -> np.ndarray:
    """VHotP reader of the reference's evaluator (…evaluator_par.py:42-46)."""
    return formats.read_vhot(fileName)


# ---------------------------------------------------------------- AllParams
def allparams_from_mapping(params_input: Sequence[Sequence[float]], template_row: Sequence[float],
                           indicator_row: Sequence[float], corrections: dict | None = None,
                           out_path: str | Path | None = None, dtype=np.float64) -> np.ndarray:
    """GA parameter vectors -> AllParams rows (extractModel_mappings.py:290-331).

    template_row: one AllParams row of the model (AllParams_reference.csv);
    indicator_row: the same row of AllParams_for_params.csv, where the value
    12300 + k marks every position that GA parameter k sets
    (create_params_to_all_params, :258-272); corrections: index -> value
    applied to every row (correction_mappings.json, :240-251).  Writes
    AllParams.csv as the reference does (the set count, then '%.5E' rows)
    when out_path is given.  Returns [n_sets, len(template_row)] of `dtype`
    (float64; float32 gives the same values rounded entry by entry, built
    without a float64 copy, as the simulator takes them)."""
    tmpl = np.asarray(template_row, dtype=np.float64)
    ind = np.asarray(indicator_row, dtype=np.float64)
    params = np.asarray(params_input, dtype=np.float64)
    if params.ndim != 2:
        raise ValueError("params_input must be [n_sets][n_params]")
    out = np.empty((params.shape[0], tmpl.size), dtype=dtype)
    out[:] = tmpl.astype(dtype)[None, :]
    for k in range(params.shape[1]):
        pos = np.nonzero(ind == PARAM_INDICATOR_BASE + k)[0]
        out[:, pos] = params[:, k:k + 1]
    for idx, v in (corrections or {}).items():
        out[:, int(idx)] = float(v)
    if out_path is not None:
        with open(out_path, "w", newline="") as fh:
            wr = csv.writer(fh)
            wr.writerow([str(params.shape[0])])
            for row in out:
                wr.writerow(["%.5E" % x for x in row])
    return out


def load_mapping(data_dir: str | Path) -> tuple[np.ndarray, np.ndarray, dict]:
    """(template_row, indicator_row, corrections) from a model's Data dir."""
    d = Path(data_dir)
    def row(name):
        lines = [ln for ln in (d / name).read_text().splitlines() if ln.strip()]
        return np.array([float(x) for x in lines[1].split(",") if x.strip()], dtype=np.float64)
    corr = {}
    if (d / "correction_mappings.json").exists():
        corr = json.loads((d / "correction_mappings.json").read_text())
    return row("AllParams_reference.csv"), row("AllParams_for_params.csv"), corr


# ---------------------------------------------------------------- features
def _peaks(v: np.ndarray, thr: float) -> np.ndarray:
    """eFEL peak_indices: the maximum of every excursion above threshold."""
    above = v >= thr
    if not above.any():
        return np.zeros(0, dtype=np.int64)
    d = np.diff(above.astype(np.int8))
    ups = list(np.nonzero(d == 1)[0] + 1)
    downs = list(np.nonzero(d == -1)[0] + 1)
    if above[0]:
        ups = [0] + ups
    if len(downs) < len(ups):
        downs.append(v.size)
    return np.array([u + int(np.argmax(v[u:e])) for u, e in zip(ups, downs)], dtype=np.int64)


def efel_features(t: np.ndarray, v: np.ndarray, stim_start: float = STIM_START, stim_end: float = STIM_END,
                  threshold: float = THRESHOLD) -> dict[str, np.ndarray | None]:
    """The eFEL features efel_ext.py requests (feature_list, :13).

    Each restates the feature's published definition in eFEL's feature
    documentation (BlueBrain eFEL, the eFeatures descriptions; the reference
    pins eFEL by git commit, GUI/requirements.txt:23, and calls it at
    P/efel_ext.py:62 with Threshold -30 mV and the default
    DerivativeThreshold 10 mV/ms):

    * voltage_base -- the mean voltage over the last 10 % of the time before
      the stimulus: mean V over [0.9 stim_start, stim_start].
    * peak_indices / peak_time -- for every excursion above Threshold (from
      an upward crossing to the next downward one, or the trace's end), the
      sample of its maximum; peak_time is its time.  Only peaks within
      [stim_start, stim_end] are kept.
    * AP_begin_indices -- for each peak, the first sample after the previous
      peak (the first: after stim_start) where dV/dt >= DerivativeThreshold
      (dV/dt by central differences, numpy.gradient).
    * AP_amplitude -- V at the peak minus V at its AP begin.
    * min_AHP_values / AHP_depth -- the minimum of V between a peak and the
      next (after the last peak: up to stim_end); AHP_depth = min_AHP_values
      - voltage_base.
    * spike_half_width -- the time between the upward and the downward
      crossing of the half level 0.5 (V_peak + V_AP_begin), each crossing
      time linearly interpolated between samples; spikes whose fall does not
      reach the half level before the trace ends are left out.
    * voltage_after_stim -- the mean voltage over [stim_end + 25 %, stim_end
      + 75 %] of the time after the stimulus.

    A feature that cannot be computed (no peak in the window; no samples) is
    None, as eFEL returns None.  tests/test_efel_features.py checks every
    definition on traces whose features follow by hand from it: no spikes,
    one spike, spikes at both window edges, two spikes."""
    t = np.asarray(t, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    out: dict[str, np.ndarray | None] = {}
    base = (t >= 0.9 * stim_start) & (t <= stim_start)
    vb = float(np.mean(v[base])) if base.any() else float("nan")
    out["voltage_base"] = np.array([vb])
    end = t[-1]
    after = (t >= stim_end + 0.25 * (end - stim_end)) & (t <= stim_end + 0.75 * (end - stim_end))
    out["voltage_after_stim"] = np.array([float(np.mean(v[after]))]) if after.any() else None
    pk = _peaks(v, threshold)
    pk = pk[(t[pk] >= stim_start) & (t[pk] <= stim_end)] if pk.size else pk
    if pk.size == 0:
        for k in ("peak_time", "AP_amplitude", "spike_half_width", "AHP_depth"):
            out[k] = None
        return out
    out["peak_time"] = t[pk]
    dvdt = np.gradient(v, t)
    begins = []
    lo = int(np.searchsorted(t, stim_start))
    for k, p in enumerate(pk):
        start = lo if k == 0 else int(pk[k - 1]) + 1
        w = np.nonzero(dvdt[start:p + 1] >= DERIVATIVE_THRESHOLD)[0]
        begins.append(start + int(w[0]) if w.size else start)
    begins = np.array(begins)
    out["AP_amplitude"] = v[pk] - v[begins]
    hi = int(np.searchsorted(t, stim_end, side="right"))
    ahp = []
    for k, p in enumerate(pk):
        e = int(pk[k + 1]) if k + 1 < pk.size else max(hi, int(p) + 1)
        ahp.append(float(np.min(v[p:e])) if e > p else float(v[p]))
    out["AHP_depth"] = np.array(ahp) - vb
    widths = []
    for b, p in zip(begins, pk):
        half = 0.5 * (v[p] + v[b])
        r = np.nonzero(v[b:p + 1] >= half)[0]
        f = np.nonzero(v[p:] < half)[0]
        if r.size == 0 or f.size == 0:
            continue
        i1 = b + int(r[0])
        i2 = p + int(f[0])
        t1 = t[i1] if i1 == b else t[i1 - 1] + (half - v[i1 - 1]) * (t[i1] - t[i1 - 1]) / (v[i1] - v[i1 - 1])
        t2 = t[i2 - 1] + (half - v[i2 - 1]) * (t[i2] - t[i2 - 1]) / (v[i2] - v[i2 - 1])
        widths.append(t2 - t1)
    out["spike_half_width"] = np.array(widths) if widths else None
    return out


def get_chi(orig_volts, volts) -> list[float]:
    """efel_ext.get_chi: mean |orig - v| per trace (sum of sqrt of squares
    over the sample count)."""
    o = np.asarray(orig_volts, dtype=np.float64)
    return [float(np.sum(np.sqrt(np.square(np.subtract(o, cv)))) / o.size) for cv in volts]


def diff_lists(lis1, lis2) -> float:
    """efel_ext.eval.diff_lists: 1000 when a feature is missing, else the RMS
    difference of the zero-padded lists."""
    if lis1 is None or lis2 is None:
        return 1000
    a, b = np.asarray(lis1, dtype=np.float64), np.asarray(lis2, dtype=np.float64)
    if a.size > b.size:
        b = np.concatenate((b, np.zeros(a.size - b.size)))
    if b.size > a.size:
        a = np.concatenate((a, np.zeros(b.size - a.size)))
    return float(np.sqrt(((a - b) ** 2).mean()))


def efel_eval(target_volts_list, data_volts_list, times,
              features: Callable = efel_features) -> list[np.ndarray]:
    """efel_ext.eval: per data trace, the seven scores of ALL_FEATURES against
    the target; NaN differences score 10000, traces holding NaN 100000."""
    data = np.asarray(data_volts_list, dtype=np.float64)
    nan_rows = np.isnan(data).any(axis=1)
    good = data[~nan_rows]
    tf = features(times, target_volts_list[0])
    chis = get_chi(target_volts_list[0], good)
    scored = []
    for i, v in enumerate(good):
        df = features(times, v)
        row = []
        for name in ALL_FEATURES:
            d = chis[i] if name == "chi" else diff_lists(tf[name], df[name])
            row.append(10000 if math.isnan(d) else d)
        scored.append(np.array(row, dtype=np.float64))
    res, k = [], 0
    for bad in nan_rows:
        if bad:
            res.append(np.zeros(len(ALL_FEATURES)) + 100000)
        else:
            res.append(scored[k])
            k += 1
    return res


# ---------------------------------------------------------------- evaluator
@dataclass
class MultiStimEvaluator:
    """neurogpu_multistim_evaluator without processes or files.

    model: a formats.ReferenceModel (morphology, stimulus site, recording);
    stims [n_stims][nt] nA; target_volts [n_stims][nt]; pmin/pmax bound the
    GA parameters (opt_table.csv rows); mapping = (template_row,
    indicator_row, corrections) as in allparams_from_mapping.  ``run`` may be
    replaced (tests), by default it is neurogpu_b200.sim.run."""
    model: "formats.ReferenceModel"
    stims: np.ndarray
    target_volts: np.ndarray
    pmin: np.ndarray
    pmax: np.ndarray
    mapping: tuple
    run: Callable | None = None
    objectives: list[str] = field(default_factory=list)

    def __post_init__(self):
        self.stims = np.ascontiguousarray(self.stims, dtype=np.float32)
        self.target_volts = np.asarray(self.target_volts, dtype=np.float64)
        if not self.objectives:
            self.objectives = [f"{f if f != 'peak_time' else 'ISI values'}_{k + 1}"
                               for k in range(self.stims.shape[0]) for f in ALL_FEATURES]
        self.times = np.cumsum(np.asarray(self.model.dts, dtype=np.float64))

    def simulate(self, param_values) -> np.ndarray:
        """V at the recording site, [n_individuals][n_stims][nt]."""
        rows = allparams_from_mapping(param_values, *self.mapping, dtype=np.float32)
        n_comps, n_file_params = self.model.cell.n_sections, rows.shape[1] // self.model.cell.n_sections
        file_params = rows.reshape(len(rows), n_file_params, n_comps)
        n_models = int(self.model.raw["basic_const"]["NModels"][0]) if self.model.raw else None
        params = formats.map_params(file_params, n_models, n_file_params) if n_models else file_params
        run = self.run
        if run is None:
            from .sim import run
        c = self.model.cell
        out = run(c, params, self.stims, self.model.dts, self.model.stim_node, self.model.stim_area,
                  np.asarray(self.model.rec_nodes[:1], dtype=np.int32), self.model.v_init)
        return np.asarray(out)[:, :, 0, :]

    def evaluate_with_lists(self, param_values) -> list[np.ndarray]:
        """Scores per individual: ALL_FEATURES for stimulus 1, then 2, ... (the
        reference's concatenation, …evaluator_par.py:239-290)."""
        v = self.simulate(param_values)
        scores = None
        for s in range(self.stims.shape[0]):
            st = efel_eval([self.target_volts[s]], v[:, s, :], self.times)
            scores = st if scores is None else [np.append(a, b) for a, b in zip(scores, st)]
        return scores
