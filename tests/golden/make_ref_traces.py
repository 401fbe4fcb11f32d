#!/usr/bin/env python
"""Runs the reference's own GPU simulator (oracle/_ref/neuroGPU_ttpc512, built
unmodified from GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src by oracle/build_ref.sh)
on its shipped 512-node TTPC model, on a GPU, and

1. checks that two runs of the same input agree bit for bit,
2. compares its traces with the oracle (FP64 and FP32, finite-difference
   conductance as in src/CudaStuff.cu:293-300) and with this library's FP32
   simulation, by spike timing and by voltage away from spikes,
3. with --save PATH, writes the traces and the parameter sets it was given
   to PATH (committed as tests/golden/ref_ttpc512_traces.npz; the parity
   tests read it),
4. with --time-sets N, times the reference and this library on the same model
   and N parameter sets: the reference's own CUDA-event figures ("solver took"
   around the kernel, "total took" around set-up + kernel + copy-back,
   src/CudaStuff.cu:487-541) against this library's kernel time (CUDA events)
   and its host-buffer ngpu_run (wall clock), as one JSON line.

Run from the repository root on a machine with a GPU; it only reads the
committed fixtures under tests/golden/ttpc512 and the prebuilt binary.

Input files follow the reference's Data/ layout (src/Util.h:44-55): the binary
runs from <tmp>/bin and reads ../Data.  Parameter sets: set 0 is the shipped
AllParams_reference.csv; set k > 0 scales every parameter row of it by its own
seeded factor in [1 - spread, 1 + spread].  The reference's compiled-in limits
bound the inputs: one stimulus (NTRACES 1) and at most 32767 sets (the block
index is a 16-bit MYDTYPE, src/CudaStuff.cu:157).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

from neurogpu_b200 import formats  # noqa: E402

FIX = HERE / "ttpc512"
BINARY = ROOT / "oracle" / "_ref" / "neuroGPU_ttpc512"
MAX_SETS = 32767


def param_sets(n_sets: int, spread: float, seed: int = 512) -> np.ndarray:
    """[n_sets, 19, 241] float32 in the file's parameter order, exactly as the
    reference parses them back from the AllParams.csv this script writes."""
    base = formats.read_params_csv(FIX / "AllParams_reference.csv", 241, 19, True)[0]
    rng = np.random.default_rng(seed)
    f = rng.uniform(1.0 - spread, 1.0 + spread, (n_sets, base.shape[0], 1))
    f[0] = 1.0
    p = (base[None] * f).astype(np.float32)
    # what the reference reads back from the '%.5E' text write_allparams_csv writes
    uniq, inv = np.unique(p.reshape(-1), return_inverse=True)
    back = np.array([formats.ref_atof(f"{x:.5E}") for x in uniq], dtype=np.float32)
    return back[inv].reshape(p.shape)


def write_run_dir(root: Path, params: np.ndarray) -> Path:
    data = root / "Data"
    (root / "bin").mkdir(parents=True)
    data.mkdir()
    for name in ("BasicConstSegP.csv", "Sim.csv", "Stim_meta.csv", "times.csv"):
        shutil.copyfile(FIX / name, data / name)
    shutil.copyfile(FIX / "Stim_raw0.csv", data / "Stim_raw.csv")   # no argv: Stim_raw.csv
    formats.write_allparams_csv(data / "AllParams.csv", params)
    return data


def run_reference(root: Path, timeout: float) -> dict:
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    t0 = time.perf_counter()
    p = subprocess.run([str(BINARY)], cwd=root / "bin", capture_output=True, text=True,
                       timeout=timeout, env=env)
    wall = time.perf_counter() - t0
    out = p.stdout + p.stderr
    if p.returncode != 0 or "ERROR: CUDA RT call" in out or "Failed to read" in out:
        raise RuntimeError(f"reference run failed (rc {p.returncode}):\n{out[-3000:]}")
    solver = float(re.search(r"solver took ([0-9.]+) ms", out).group(1))
    total = float(re.search(r"total took ([0-9.]+) ms", out).group(1))
    v = formats.read_vhot(root / "Data" / "VHotP0.dat")
    return {"vhot": v, "solver_ms": solver, "total_ms": total, "wall_s": wall}


def reference_traces(params: np.ndarray, timeout: float) -> tuple[np.ndarray, dict]:
    with tempfile.TemporaryDirectory(prefix="ngpu_ref_") as tmp:
        root = Path(tmp)
        write_run_dir(root, params)
        r1 = run_reference(root, timeout)
        os.remove(root / "Data" / "VHotP0.dat")
        r2 = run_reference(root, timeout)
    n_sets = params.shape[0]
    nt = r1["vhot"].size // n_sets
    tr1 = r1["vhot"].reshape(n_sets, nt)
    tr2 = r2["vhot"].reshape(n_sets, nt)
    info = {"deterministic": bool(np.array_equal(tr1, tr2)),
            "max_run_to_run_mv": float(np.max(np.abs(tr1 - tr2))),
            "solver_ms": r1["solver_ms"], "total_ms": r1["total_ms"]}
    return tr1.astype(np.float32), info


def model_inputs():
    return formats.read_data_dir(FIX, stim_index=0, params_file="AllParams_reference.csv")


def compare(ref: np.ndarray, params: np.ndarray, with_product: bool) -> dict:
    import oracle_py
    from helpers import spike_time_error, subthreshold_error
    m = model_inputs()
    c = m.cell
    dt = float(m.dts[0])
    res = {}
    runs = {}
    for prec in ("f64", "f32"):
        runs["oracle_" + prec] = oracle_py.run(
            c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask, params,
            m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init, precision=prec, fd=True)[:, 0, 0]
    if with_product:
        from neurogpu_b200.sim import run
        runs["product_fp32"] = run(c, params, m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes,
                                   m.v_init)[:, 0, 0].astype(np.float64)
    ref64 = ref.astype(np.float64)
    for name, got in runs.items():
        st, mism = spike_time_error(got[:, None, None], ref64[:, None, None], dt)
        res[name] = {"spike_time_ms": st, "spike_count_mismatches": mism,
                     "subthreshold_mv": subthreshold_error(got[:, None, None], ref64[:, None, None], dt),
                     "max_abs_mv": float(np.max(np.abs(got - ref64)))}
    return res


def time_both(n_sets: int, spread: float, timeout: float) -> dict:
    import torch
    from neurogpu_b200.sim import Model, Simulator, run
    params = param_sets(n_sets, spread)
    with tempfile.TemporaryDirectory(prefix="ngpu_ref_") as tmp:
        root = Path(tmp)
        write_run_dir(root, params)
        r = run_reference(root, timeout)
    m = model_inputs()
    c = m.cell
    nt = m.amps.shape[1]
    units = float(c.n_nodes) * nt * n_sets
    model = Model(c)
    sim = Simulator(model, n_sets, 1)
    sim.set_params(params)
    sim.set_stimulus(m.amps, m.dts, m.stim_node, m.stim_area)
    sim.set_recording(m.rec_nodes)
    stream = torch.cuda.current_stream()
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        sim.init(m.v_init, stream)
        sim.advance(0, nt, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    sim.close()
    walls = []
    for _ in range(2):
        t0 = time.perf_counter()
        run(model, params, m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init)
        walls.append(time.perf_counter() - t0)
    model.close()
    return {"workload": f"TTPC 512-node shipped model x {n_sets} parameter sets, {nt} steps",
            "compartment_steps": units,
            "reference_solver_ms": r["solver_ms"], "reference_total_ms": r["total_ms"],
            "reference_solver_cs_per_s": units / (r["solver_ms"] * 1e-3),
            "reference_total_cs_per_s": units / (r["total_ms"] * 1e-3),
            "ours_kernel_ms": best, "ours_kernel_cs_per_s": units / (best * 1e-3),
            "ours_ngpu_run_wall_ms": min(walls) * 1e3,
            "ours_ngpu_run_cs_per_s": units / min(walls),
            "kernel_speedup": r["solver_ms"] / best,
            "total_speedup": r["total_ms"] / (min(walls) * 1e3)}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--sets", type=int, default=16)
    ap.add_argument("--spread", type=float, default=0.2)
    ap.add_argument("--save", default="")
    ap.add_argument("--no-product", action="store_true")
    ap.add_argument("--time-sets", type=int, default=0)
    ap.add_argument("--timeout", type=float, default=600.0)
    ap.add_argument("--json", default="")
    a = ap.parse_args()
    if not BINARY.exists():
        print("oracle/_ref/neuroGPU_ttpc512 is not built (oracle/build_ref.sh)", file=sys.stderr)
        return 2
    if not (1 <= a.sets <= MAX_SETS and 0 <= a.time_sets <= MAX_SETS):
        print(f"set counts must lie in 1..{MAX_SETS}", file=sys.stderr)
        return 2
    params = param_sets(a.sets, a.spread)
    ref, info = reference_traces(params, a.timeout)
    info["sets"] = a.sets
    info["vs"] = compare(ref, params, not a.no_product)
    if a.save:
        np.savez_compressed(a.save, params=params, traces=ref,
                            spread=np.float32(a.spread))
    out = {"parity": info}
    if a.time_sets:
        out["timing"] = time_both(a.time_sets, a.spread, a.timeout)
    line = json.dumps(out)
    print(line)
    if a.json:
        Path(a.json).write_text(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
