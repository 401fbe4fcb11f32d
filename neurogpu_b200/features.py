"""Batched spike / ISI / amplitude / AHP / voltage features of many traces
at once on the GPU (torch tensors; CPU tensors work too).

The reference scores traces one at a time on a CPU pool (P/efel_ext.py with
eFEL, GUI/score_functions.py); a GA over thousands of individuals per
generation needs the features of all traces in one pass, and the surrogate
network is trained to predict exactly this vector.  Spikes are upward
crossings of -20 mV inside the stimulus window; every feature has a defined
value without spikes (stated per feature) so the vector is always finite.

These 20 are this project's own definitions (the surrogate's target vector),
modelled on eFEL features (the eFEL feature documentation, BlueBrain eFEL;
the reference pins its version at GUI/requirements.txt:23) but not equal to
them; the evaluator's eFEL features proper are neurogpu_b200.evaluator.
efel_features.  Correspondence, and where they differ:

  spike_count           eFEL Spikecount (eFEL counts peaks; here crossings)
  first_spike_latency   time_to_first_spike (eFEL: to the peak; here to the
                        first sample at or above threshold)
  mean_isi, isi_cv      mean of ISI_values, ISI_CV (ISIs between crossings)
  first_isi, last_isi   ISI_values[0], ISI_values[-1]
  adaptation            last ISI / first ISI (eFEL's adaptation_index is a
                        normalised average of consecutive ISI differences)
  ap_peak_mean, _std    mean and std of peak_voltage (the maximum between
                        consecutive crossings)
  ahp_mean              mean of min_AHP_values (the minimum between
                        consecutive crossings, the last to the window end)
  ap_amplitude_mean     ap_peak_mean - ahp_mean (eFEL's AP_amplitude is
                        peak - AP begin voltage)
  time_above_half       the mean time per spike above the half level between
                        those means (eFEL's spike_half_width uses each AP's
                        own begin voltage)
  voltage_base          mean V over the 10 ms before stim_on (eFEL: the last
                        10 % of the time before the stimulus)
  steady_state          mean V over the last 50 ms of the stimulus
                        (eFEL steady_state_voltage_stimend: the last 10 %)
  voltage_after_stim    mean V from stim_off + 10 ms to the trace's end
                        (eFEL: stim_off + 25 % .. 75 % of the remaining time)
  v_max, v_min_stim, v_mean_stim, v_std_stim, last_spike_time
                        maximum_voltage (whole trace), minimum_voltage,
                        mean and std of V in the window, the last crossing
"""
from __future__ import annotations

import torch

FEATURES = ("spike_count", "first_spike_latency", "mean_isi", "isi_cv", "first_isi", "last_isi",
            "adaptation", "ap_peak_mean", "ap_peak_std", "ahp_mean", "ap_amplitude_mean", "time_above_half",
            "voltage_base", "steady_state", "voltage_after_stim", "v_max", "v_min_stim", "v_mean_stim",
            "v_std_stim", "last_spike_time")
N_FEATURES = len(FEATURES)
THRESHOLD = -20.0


def extract(v: torch.Tensor, dt: float, stim_on: float, stim_off: float) -> torch.Tensor:
    """v [B, T] mV sampled every dt ms -> features [B, 20] (float32).

    Without spikes: latency, ISIs and last spike time = stimulus duration,
    cv 0, adaptation 1, peak / AHP / amplitude from the window's max / min,
    time above half 0."""
    v = v.float()
    B, T = v.shape
    dev = v.device
    i_on, i_off = int(round(stim_on / dt)), min(T, int(round(stim_off / dt)))
    dur = (i_off - i_on) * dt
    w = v[:, i_on:i_off]
    up = (w[:, :-1] < THRESHOLD) & (w[:, 1:] >= THRESHOLD)          # [B, W-1]
    n = up.sum(1).float()
    has1, has2 = n >= 1, n >= 2
    idx = torch.arange(up.shape[1], device=dev, dtype=torch.float32)
    tcross = (idx + 1.0)[None, :] * dt                               # time of the sample at/after the crossing
    big = torch.full_like(tcross.expand(B, -1), 1e9)
    first = torch.where(up, tcross, big).min(1).values
    last = torch.where(up, tcross, -big).max(1).values
    first_lat = torch.where(has1, first, torch.full_like(first, dur))
    last_t = torch.where(has1, last, torch.full_like(last, dur))
    # ISIs from consecutive crossings: rank the crossings, take differences
    rank = torch.cumsum(up.to(torch.int32), 1)
    t_sorted = torch.sort(torch.where(up, tcross, big), 1).values    # crossing times ascending, then 1e9
    kmax = int(n.max().item()) if B else 0
    kmax = max(kmax, 2)
    ts = t_sorted[:, :kmax]
    valid = ts < 1e8
    isi = ts[:, 1:] - ts[:, :-1]
    iv = valid[:, 1:] & valid[:, :-1]
    n_isi = iv.sum(1).float()
    isi_sum = torch.where(iv, isi, torch.zeros_like(isi)).sum(1)
    mean_isi = torch.where(has2, isi_sum / n_isi.clamp(min=1), torch.full_like(n, dur))
    isi_sq = torch.where(iv, (isi - mean_isi[:, None]) ** 2, torch.zeros_like(isi)).sum(1)
    isi_cv = torch.where(has2, torch.sqrt(isi_sq / n_isi.clamp(min=1)) / mean_isi.clamp(min=1e-6), torch.zeros_like(n))
    first_isi = torch.where(has2, isi[:, 0], torch.full_like(n, dur))
    last_pos = (n_isi - 1).clamp(min=0).long()
    last_isi = torch.where(has2, isi.gather(1, last_pos[:, None])[:, 0], torch.full_like(n, dur))
    adaptation = torch.where(has2, last_isi / first_isi.clamp(min=1e-6), torch.ones_like(n))
    # AP peaks: max of V between consecutive crossings (segment ids from the crossing rank)
    seg = torch.cat([torch.zeros(B, 1, dtype=torch.int32, device=dev), rank], 1)   # [B, W]
    in_ap = seg > 0
    segc = seg.clamp(max=kmax).long()
    neg = torch.full((B, kmax + 1), -1e9, device=dev)
    peaks = neg.scatter_reduce(1, segc, torch.where(in_ap, w, torch.full_like(w, -1e9)), reduce="amax")[:, 1:]
    pos = torch.full((B, kmax + 1), 1e9, device=dev)
    troughs = pos.scatter_reduce(1, segc, torch.where(in_ap, w, torch.full_like(w, 1e9)), reduce="amin")[:, 1:]
    pv = valid & (peaks > -1e8)
    npk = pv.sum(1).float().clamp(min=1)
    pk_mean = torch.where(has1, torch.where(pv, peaks, torch.zeros_like(peaks)).sum(1) / npk, w.max(1).values)
    pk_std = torch.where(has1, torch.sqrt(torch.where(pv, (peaks - pk_mean[:, None]) ** 2,
                                                      torch.zeros_like(peaks)).sum(1) / npk), torch.zeros_like(n))
    ahp_mean = torch.where(has1, torch.where(pv, troughs, torch.zeros_like(troughs)).sum(1) / npk, w.min(1).values)
    amp = pk_mean - ahp_mean
    half = 0.5 * (pk_mean + ahp_mean)
    above = ((w >= half[:, None]) & in_ap).sum(1).float() * dt
    t_half = torch.where(has1, above / n.clamp(min=1), torch.zeros_like(n))
    def mean_win(a, b):
        ia, ib = max(0, int(round(a / dt))), min(T, max(int(round(a / dt)) + 1, int(round(b / dt))))
        return v[:, ia:ib].mean(1)
    vb = mean_win(max(0.0, stim_on - 10.0), stim_on)
    ss = mean_win(max(stim_on, stim_off - 50.0), stim_off)
    after = mean_win(stim_off + 10.0, T * dt) if stim_off + 10.0 < T * dt else v[:, -1]
    return torch.stack([n, first_lat, mean_isi, isi_cv, first_isi, last_isi, adaptation, pk_mean, pk_std, ahp_mean,
                        amp, t_half, vb, ss, after, v.max(1).values, w.min(1).values, w.mean(1), w.std(1),
                        last_t], 1)


def extract_device(v: torch.Tensor, dt: float, stim_on: float, stim_off: float,
                   threshold: float = THRESHOLD) -> torch.Tensor:
    """extract() by the library's CUDA kernel (ngpu_trace_features): v [B, T]
    float32 on the GPU, any strides; one thread per trace, both passes over
    the trace in one launch."""
    import ctypes as C

    from . import _ffi
    if not v.is_cuda or v.dtype != torch.float32 or v.dim() != 2:
        raise ValueError("v must be a float32 CUDA tensor [B, T]")
    B, T = v.shape
    out = torch.empty((B, N_FEATURES), dtype=torch.float32, device=v.device)
    stream = torch.cuda.current_stream(v.device).cuda_stream
    _ffi.check("ngpu_trace_features", _ffi.lib().ngpu_trace_features(
        C.c_void_p(v.data_ptr()), v.stride(0), v.stride(1), B, T, float(dt), float(stim_on), float(stim_off),
        float(threshold), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out
