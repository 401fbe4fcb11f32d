"""FP64 oracle fixtures for the long-run parity tests (tests/test_long_runs.py).

Each benchmark configuration is run by the CPU oracle (oracle/oracle.c, the
FP64 restatement of the reference's step, GUI/BBP_TTPC_EXAMPLE/
pyNeuroGPU_unix/src/CudaStuff.cu:142-335) at its stated duration on a
deterministic sample of its parameter sets:

  hh_500ms      config 2: the 500-compartment HH-type cell, 1024 sets x 3
                protocols, 500 ms (20,000 steps); 16 sets spread over the batch
  ttpc_2000ms   config 3: the 1501-compartment TTPC-like cell, 4096 sets x 3
                protocols, 2000 ms (80,000 steps); 8 sets spread over the batch
  uneven_500ms  config 4: the uneven batch (200/800/1500/3000-compartment
                HH-type trees, 2048 sets each) x 5 protocols, 500 ms; a 1 %
                sample of the 8192 sets (82), drawn per tree with a seeded rng

Stored per configuration (float32 voltages, float64 spike times):
  sets      [n]           sampled set indices (uneven: index within its tree)
  tree      [n]           uneven only: the tree (index into the sizes) of each set
  v         [n, n_stim, n_sub]  soma V every `stride` steps (1 ms)
  spk, spk_off            upward -20 mV crossings of the full-resolution
                          trace, linearly interpolated (ms), flattened over
                          the [n, n_stim] traces in C order, with offsets
The GPU test runs the whole batch and compares these sets.  The sampled
voltages are the oracle's float64 values rounded to float32 (4e-6 mV at
100 mV), far below the 0.1 mV bound they are checked against.

The model's own sensitivity, for configs 2 and 3: the same sampled sets
rerun by the FP64 oracle with every parameter nudged by one part in 1e7
(about one float32 ulp; a seeded random sign per value, rounded to float32),
and by the oracle's float32 build, each compared with the FP64 run as the
GPU run is (sens_* and f32_*: spike_ms, mismatches, dv_away_mV at the 1 ms
samples).  A model whose spike times move this far under perturbations at
float32 rounding scale cannot be followed more closely by any float32
arithmetic.

Run: python tests/golden/make_long_runs.py [--only name] [--sensitivity]
(about 8 minutes on 8 cores, 3 more with --sensitivity; the oracle is
OpenMP-parallel over instances).
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE.parent))

STRIDE = 40          # 1 ms at dt = 0.025 ms
OUT = HERE / "long_runs.npz"


def sample_spread(n_total: int, n: int) -> np.ndarray:
    return np.unique(np.round(np.linspace(0, n_total - 1, n)).astype(np.int64))


def uneven_sample(per_tree: int, n_trees: int, frac: float = 0.01, seed: int = 11) -> list[np.ndarray]:
    """frac of all sets, split over the trees (the remainder to the first
    trees), drawn without replacement per tree, sorted."""
    total = int(round(frac * per_tree * n_trees))
    rng = np.random.default_rng(seed)
    counts = [total // n_trees + (1 if k < total % n_trees else 0) for k in range(n_trees)]
    return [np.sort(rng.choice(per_tree, size=c, replace=False)) for c in counts]


def workloads():
    """name -> list of (workload restricted to the sample, sampled set indices, tree index)."""
    from neurogpu_b200 import configs
    hh = configs.hh_active(n_sets=1024, t_stop=500.0)
    tt = configs.ttpc_like(n_sets=4096, t_stop=2000.0)
    ub = configs.uneven_batch(n_sets=8192, t_stop=500.0)
    out = {
        "hh_500ms": [(hh, sample_spread(1024, 16), 0)],
        "ttpc_2000ms": [(tt, sample_spread(4096, 8), 0)],
        "uneven_500ms": [(w, idx, k) for k, (w, idx) in enumerate(zip(ub, uneven_sample(ub[0].n_sets, len(ub))))],
    }
    return out


def summarise(traces: np.ndarray, dt: float):
    """(subsampled float32 voltages, flat spike times, offsets) of traces [n, n_stim, nt]."""
    from helpers import spike_times
    n, ns, nt = traces.shape
    v = traces[:, :, ::STRIDE].astype(np.float32)
    spk, off = [], [0]
    for tr in traces.reshape(n * ns, nt):
        s = spike_times(tr, dt)
        spk.append(s)
        off.append(off[-1] + s.size)
    return v, (np.concatenate(spk) if spk else np.zeros(0)), np.asarray(off, dtype=np.int64)


SENS_EPS = 1e-7


def perturbed(w, eps: float = SENS_EPS, seed: int = 1):
    """w with every parameter multiplied by 1 +- eps (seeded signs), in float32."""
    from dataclasses import replace
    rng = np.random.default_rng(seed)
    p = w.params.astype(np.float64) * (1.0 + eps * rng.choice([-1.0, 1.0], w.params.shape))
    return replace(w, params=p.astype(np.float32))


def deviation(a: np.ndarray, b: np.ndarray, dt: float, window_ms: float = 2.0, stride: int = 1):
    """(max spike-time difference over matched spikes, spike-count
    mismatches, max |a - b| farther than window_ms from any spike) of traces
    [..., nt], at every stride-th sample."""
    from helpers import spike_times
    a2, b2 = a.reshape(-1, a.shape[-1]), b.reshape(-1, b.shape[-1])
    win = int(round(window_ms / dt))
    worst_t, mism, worst_v = 0.0, 0, 0.0
    for x, y in zip(a2, b2):
        sx, sy = spike_times(x, dt), spike_times(y, dt)
        if sx.size != sy.size:
            mism += 1
        elif sx.size:
            worst_t = max(worst_t, float(np.max(np.abs(sx - sy))))
        keep = np.ones(x.size, dtype=bool)
        for t in np.concatenate([sx, sy]):
            k = int(t / dt)
            keep[max(0, k - win):k + win + 1] = False
        keep[np.arange(x.size) % stride != 0] = False
        if keep.any():
            worst_v = max(worst_v, float(np.max(np.abs(x[keep] - y[keep]))))
    return worst_t, mism, worst_v


def sensitivity(name: str, data: dict):
    import oracle_py
    (w, idx, _), = workloads()[name]
    ws = w.take(idx)
    ref = oracle_py.run_workload(ws)[:, :, 0, :]
    per = oracle_py.run_workload(perturbed(ws))[:, :, 0, :]
    t, mism, v = deviation(per, ref, ws.dt, stride=STRIDE)
    data[f"{name}/sens_eps"] = np.float64(SENS_EPS)
    data[f"{name}/sens_spike_ms"] = np.float64(t)
    data[f"{name}/sens_mismatches"] = np.int64(mism)
    data[f"{name}/sens_dv_away_mV"] = np.float64(v)
    print(f"{name}: parameters x (1 +- {SENS_EPS:g}): spikes move {t:.4f} ms, {mism} count changes, "
          f"{v:.4f} mV away from spikes", flush=True)
    # the oracle's float32 build (storage and channel arithmetic in float32,
    # libm's correctly rounded functions) against its float64 build
    f32 = oracle_py.run_workload(ws, precision="f32")[:, :, 0, :]
    t, mism, v = deviation(f32, ref, ws.dt, stride=STRIDE)
    data[f"{name}/f32_spike_ms"] = np.float64(t)
    data[f"{name}/f32_mismatches"] = np.int64(mism)
    data[f"{name}/f32_dv_away_mV"] = np.float64(v)
    print(f"{name}: the oracle's float32 build: spikes {t:.4f} ms, {mism} count changes, "
          f"{v:.4f} mV away from spikes", flush=True)


def main():
    import oracle_py
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--sensitivity", action="store_true", help="only the sensitivity runs of configs 2 and 3")
    args = ap.parse_args()
    data = dict(np.load(OUT)) if OUT.exists() else {}
    data["stride"] = np.int64(STRIDE)
    if args.sensitivity:
        for name in ("hh_500ms", "ttpc_2000ms"):
            if not args.only or name == args.only:
                sensitivity(name, data)
        np.savez_compressed(OUT, **data)
        return
    for name, parts in workloads().items():
        if args.only and name != args.only:
            continue
        t0 = time.time()
        vs, spks, offs, sets, trees = [], [], [], [], []
        base = 0
        for w, idx, k in parts:
            ws = w.take(idx)
            ref = oracle_py.run_workload(ws)[:, :, 0, :]  # soma, [n, n_stim, nt]
            v, spk, off = summarise(ref, ws.dt)
            vs.append(v)
            spks.append(spk)
            offs.append(off[:-1] + base)
            base += spk.size
            sets.append(idx)
            trees.append(np.full(idx.size, k, dtype=np.int64))
        data[f"{name}/v"] = np.concatenate(vs)
        data[f"{name}/spk"] = np.concatenate(spks)
        data[f"{name}/spk_off"] = np.concatenate(offs + [np.array([base], dtype=np.int64)])
        data[f"{name}/sets"] = np.concatenate(sets)
        data[f"{name}/tree"] = np.concatenate(trees)
        n_spk = data[f"{name}/spk"].size
        print(f"{name}: {data[f'{name}/v'].shape} samples, {n_spk} spikes, {time.time() - t0:.0f} s", flush=True)
        np.savez_compressed(OUT, **data)


if __name__ == "__main__":
    main()
