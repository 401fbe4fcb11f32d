#!/usr/bin/env python
"""Benchmark: compartment-steps/s of the batched neuron simulation on B200.

Workload (``ttpc_like``): a seeded ~1500-compartment thick-tufted pyramidal
morphology with the 13-mechanism TTPC channel set, 4096 parameter sets x 3
stimulus protocols = 12288 instances, dt = 0.025 ms (the 2000 ms protocol is
80000 steps).  One bench "step" is one pass of the hot path over the whole
batch for ``--chunk`` timesteps (default 800 = 20 ms of simulated time),
continuing from the resident state of the previous step.

Timing: W untimed warm-up steps, then exactly K steps between barriers and
device syncs, timed with CUDA events on the launching stream; max over
ranks.  The simulation state (>400 MB) is larger than L2, so every step
streams it from HBM.  ``--gpus N`` runs one process per GPU (torchrun), each
rank its own 12288-instance batch (weak scaling, no data-path collective).

``--impl reference`` times the reference's CPU path for the same
configuration.  The reference has no usable CPU implementation of this path
(its serial path is compiled out and calls an undefined function), so the
CPU restatement in oracle/ (FP64, OpenMP over all host threads) stands in.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "compartment-steps/s (TTPC-like x4096)"
UNIT = "compartment-steps/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_FILE = ROOT / "profiles" / "ngpu_jit_advance_ttpc_like_x4096.md"
# the other model family, for profiling (--model hh_active): its own metric name and ncu summary
UNEVEN_TRAFFIC_FILE = ROOT / "profiles" / "ngpu_jit_batch_advance_uneven_x8192.md"
MODELS = {"ttpc_like": (METRIC, TRAFFIC_FILE),
          "hh_active": ("compartment-steps/s (HH 500-compartment x4096)",
                        ROOT / "profiles" / "ngpu_jit_advance_hh_x4096.md")}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ngpu", choices=["ngpu", "reference"])
    ap.add_argument("--chunk", type=int, default=800,
                    help="timesteps per bench step (uneven_batch: per launch within the run's graph)")
    ap.add_argument("--uneven-ms", type=float, default=500.0, help="uneven_batch: simulated ms per bench step")
    ap.add_argument("--uneven-sets", type=int, default=8192, help="uneven_batch: parameter sets over the four trees")
    ap.add_argument("--n-sets", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=2000, help="timesteps of the end-to-end run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-sets", type=int, default=64)
    ap.add_argument("--cpu-sample-steps", type=int, default=800)
    ap.add_argument("--ga-pop", type=int, default=8192)
    ap.add_argument("--ga-gens", type=int, default=20)
    ap.add_argument("--ga-fits", type=int, default=3, help="ga: targets fitted (the line reports the median)")
    ap.add_argument("--ga-train", type=int, default=200_000, help="ga: the surrogate's training simulations")
    ap.add_argument("--ga-epochs", type=int, default=30)
    ap.add_argument("--model", default="ttpc_like", choices=sorted(MODELS),
                    help="the cell of the default workload: the TTPC-like headline, or the HH-type cell")
    ap.add_argument("--workload", default="ttpc_like", choices=["ttpc_like", "uneven_batch", "ga", "ga_ops", "gemm", "explore"],
                    help="uneven_batch: 8192 sets over 200/800/1500/3000-compartment trees x 5 protocols, "
                         "one launch per chunk, the run captured as a CUDA graph (auxiliary line)")
    return ap.parse_args()


def workload(n_sets: int, model: str = "ttpc_like"):
    """The TTPC-like headline workload (2000 ms), or the HH-type cell of the
    other model family (500 compartments, 500 ms) for profiling."""
    from neurogpu_b200 import configs
    if model == "hh_active":
        return configs.hh_active(n_sets=n_sets)
    return configs.ttpc_like(n_sets=n_sets)


def hbm_peak():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_comp_step_file(path: Path):
    """DRAM bytes per compartment-step of an advance kernel from a committed
    ncu summary (dram__bytes_read.sum + dram__bytes_write.sum)."""
    try:
        m = re.search(r"traffic_bytes_per_compartment_step:\s*([0-9.eE+-]+)", path.read_text())
        return float(m.group(1)) if m else None
    except Exception:
        return None


def traffic_per_comp_step(model: str = "ttpc_like"):
    return traffic_per_comp_step_file(MODELS[model][1])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over the ranks (a CUDA tensor under NCCL, a host one
    otherwise)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_rate(units_per_rank: float, seconds: float, world: int) -> tuple[float, float]:
    """Whole-job rate of N replicas: every rank processed units_per_rank in
    its own time, and the job lasts as long as the slowest rank.  Returns
    (units of all ranks / slowest time, slowest time)."""
    t = max_over_ranks(seconds, world)
    return units_per_rank * world / t, t


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _oracle_rate(sub, threads: int, precision: str) -> tuple[float, float]:
    """(compartment-steps/s, seconds) of one oracle run of workload `sub`."""
    import oracle_py
    t = time.perf_counter()
    oracle_py.run_workload(sub, precision=precision, n_threads=threads)
    el = time.perf_counter() - t
    return sub.compartment_steps() / el, el


def cpu_baseline(w, n_sets: int, n_steps: int) -> dict:
    """The oracle (the C restatement of the reference's step, OpenMP over
    instances) on bounded samples of the same workload: FP64 on every host
    thread (the value), the FP32 build on every thread, and FP64 on one
    thread."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py
    sub = w.subset(n_sets=n_sets, nt=n_steps)
    threads = os.cpu_count() or 1
    oracle_py.run_workload(sub.subset(n_sets=1, n_stim=1, nt=10), n_threads=threads)  # warm
    v64, el64 = _oracle_rate(sub, threads, "f64")
    v32, el32 = _oracle_rate(sub, threads, "f32")
    one = w.subset(n_sets=1, nt=n_steps)
    v1, el1 = _oracle_rate(one, 1, "f64")
    cs = sub.compartment_steps()
    return {"value": v64, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sub.n_sets} sets x {sub.n_stim} stimuli x {n_steps} steps of the same "
                      f"{w.cell.n_nodes}-compartment model ({cs:.3e} compartment-steps, {el64:.1f} s, FP64)",
            "fp32_all_cores": {"value": v32, "seconds": el32, "sample": "the same sample, FP32 build"},
            "fp64_one_core": {"value": v1, "seconds": el1, "cores": 1,
                              "sample": f"1 set x {one.n_stim} stimuli x {n_steps} steps, FP64"}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(args.n_sets, args.model)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py
    # bounded sample per step: a few instances x a short window, all host threads
    n_sets = max(1, threads // w.n_stim)
    sub = w.subset(n_sets=n_sets, nt=args.cpu_sample_steps)
    for _ in range(args.warmup):
        oracle_py.run_workload(sub.subset(nt=20), n_threads=threads)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        oracle_py.run_workload(sub, n_threads=threads)
        times.append(time.perf_counter() - t)
    el = float(np.mean(times))
    v = sub.compartment_steps() / el
    line = {
        "metric": MODELS[args.model][0], "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": args.model, "n_nodes": w.cell.n_nodes, "n_sets": sub.n_sets,
                   "n_stim": w.n_stim, "dt_ms": w.dt, "timesteps_per_step": sub.nt,
                   "sample_of": f"{args.n_sets} sets x {w.n_stim} protocols (rate per compartment-step)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sub.n_sets} sets x {sub.n_stim} stimuli x {sub.nt} steps per step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_uneven(args):
    """Config-4 line: the uneven batch (8192 sets over 200/800/1500/3000-
    compartment HH-type trees x 5 protocols), autotuned warps and items per
    warp per morphology.  One bench step is the whole run -- init and every
    `--chunk`-step launch of the 500 ms protocols (20,000 steps) -- captured
    once as a CUDA graph and replayed.  Warm-up: `--warmup` replays of a
    400-step graph, then one untimed run of the full graph (its capture).
    Inputs are resident; the state exceeds L2."""
    import torch
    from neurogpu_b200 import _ffi, autotune, configs
    from neurogpu_b200.sim import Batch, Model, Simulator
    rank, world, local = dist_setup(args.gpus)
    ws = configs.uneven_batch(n_sets=args.uneven_sets, t_stop=args.uneven_ms)
    sims, tuned = [], {}
    for w in ws:
        m = Model(w.cell)
        res = autotune.tune_warps(m, w.params, w.amps, w.dts, w.stim_node, w.stim_area, w.rec_nodes, w.v_init,
                                  candidates=(2, 4, 6, 8), steps=min(100, w.nt - 20), warmup=20)
        tuned[w.cell.n_nodes] = [res["n_warps"], res["items_per_warp"]]
        s = Simulator(m, w.n_sets, w.n_stim, "fp32", n_warps=res["n_warps"], items_per_warp=res["items_per_warp"])
        s.set_params(w.params)
        s.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
        s.set_recording(w.rec_nodes, 1)
        sims.append(s)
    batch = Batch(sims)
    stream = torch.cuda.Stream()
    nt = ws[0].nt
    chunk = min(args.chunk, nt)
    for _ in range(args.warmup):
        batch.run_graph(ws[0].v_init, min(400, nt), chunk, stream)
    batch.run_graph(ws[0].v_init, nt, chunk, stream)  # captures the full run's graph
    stream.synchronize()
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    _ffi.lib().ngpu_launch_count(1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        batch.run_graph(ws[0].v_init, nt, chunk, stream)
    ev1.record(stream)
    stream.synchronize()
    launches = int(_ffi.lib().ngpu_launch_count(0))
    clk = clocks.stop() if clocks else None
    cs_step = sum(w.cell.n_nodes * w.n_sets * w.n_stim for w in ws) * nt
    rate, el_s = weak_scaling_rate(cs_step * args.steps, ev0.elapsed_time(ev1) / 1e3, world)
    el_ms = el_s * 1e3
    bad = sum(s.n_bad() for s in sims)
    # roofline: bytes per compartment-step as in the default line (algorithmic,
    # or the DRAM bytes ncu measured for the batch kernel where fewer)
    peak, peak_kind = hbm_peak()
    bc = sum(w.cell.algorithmic_bytes_per_step() * w.n_sets * w.n_stim for w in ws) / \
        sum(w.cell.n_nodes * w.n_sets * w.n_stim for w in ws)
    tpcs = traffic_per_comp_step_file(UNEVEN_TRAFFIC_FILE)
    bytes_cs = bc if tpcs is None else min(bc, tpcs)
    ach = bytes_cs * cs_step * args.steps / el_s / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": f"compartment-steps/s (uneven batch x{args.uneven_sets}, 5 protocols)", "value": rate,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "uneven_batch", "trees": [w.cell.n_nodes for w in ws],
                       "sets_per_tree": ws[0].n_sets, "protocols": ws[0].n_stim, "timesteps_per_step": nt,
                       "simulated_ms_per_step": nt * ws[0].dt, "launch_chunk": chunk,
                       "warps_and_items_per_warp": tuned,
                       "graph": "init + every chunk of the run, one graph, replayed once per step",
                       "l2": "state larger than L2 (no flush)"},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_source": peak_kind, "bytes_per_compartment_step": bytes_cs,
                         "algorithmic_bytes_per_compartment_step": bc, "dram_bytes_per_compartment_step": tpcs,
                         "traffic": None if tpcs is None else tpcs * cs_step * args.steps,
                         "note": "graph time (all launches of the run), not one launch"},
            "gpu_launches": launches, "clocks": clk, "non_finite_instances": bad}))
    batch.close()


EXPLORE_BASELINE = 3.83e8  # compartment-steps/s of the reference's exploration run (RunTimes.csv)


def run_explore(args):
    """Exploration line: the reference's parameter-exploration run
    (GUI/run_neuroGPU.py, GUI/plot_param_explor.py) on its own shipped model,
    the 512-compartment BBP TTPC cell of GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/
    Data (tests/golden/ttpc512): the 100 x 100 grid over GA parameters 0 and 2
    of its opt_table.csv (10,000 sets), 3168 steps of 0.1 ms under
    Stim_raw0.csv, and every trace's dV/dt peak-count score, computed where
    the trace lies.  One bench step = init + every step of the run + the
    score, parameters resident (device-timed).  e2e: explore.explore() from
    the host grid to the host score map (AllParams rows built and uploaded,
    scores read back).  vs_baseline: the reference's RunTimes.csv for this
    run, 10,000 sets in 42,307.5 ms (init + H2D + kernel + D2H on its GPU)
    = 3.83e8 compartment-steps/s."""
    import torch
    from neurogpu_b200 import _ffi, evaluator, explore, formats
    rank, world, local = dist_setup(args.gpus)
    from neurogpu_b200.mechsets import TTPC
    d = ROOT / "tests" / "golden" / "ttpc512"
    m = formats.read_data_dir(d, stim_index=0, params_file="AllParams_reference.csv")
    # the shipped AllParams_for_params.csv marks GA parameters at entries that do
    # not match opt_table.csv's names; parameter 0 is g_pas in every section and
    # parameter 2 the soma's gNaTs2_t here
    tmpl, _, _ = evaluator.load_mapping(d)
    nc = m.cell.n_sections
    nats = tmpl.reshape(-1, nc)[TTPC.param_index("gNaTs2_tbar_NaTs2_t")]
    mapping = explore.mapping_for(tmpl, nc, {0: (TTPC.param_index("g_pas"), None),
                                             2: (TTPC.param_index("gNaTs2_tbar_NaTs2_t"),
                                                 np.nonzero(nats == nats.max())[0])})
    _, _, _, base = explore.read_opt_table(d / "opt_table.csv")
    grid = explore.gen_params(base)
    sim, score_dt = explore.grid_simulation(m, mapping, grid)
    nt = int(m.amps.shape[1])
    chunk = min(args.chunk, nt)

    def one_run():
        sim.init(m.v_init)
        for t0 in range(0, nt, chunk):
            sim.advance(t0, min(chunk, nt - t0))
        return sim.dvdt_peaks(score_dt)

    for _ in range(args.warmup):
        one_run()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    _ffi.lib().ngpu_launch_count(1)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        counts = one_run()
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = int(_ffi.lib().ngpu_launch_count(0))
    clk = clocks.stop() if clocks else None
    cs_step = len(grid) * m.cell.n_nodes * nt
    rate, el_s = weak_scaling_rate(cs_step * args.steps, ev0.elapsed_time(ev1) / 1e3, world)
    bad = sim.n_bad()
    c = counts.cpu().numpy()
    # the score kernel alone (the run's trace buffer in place): 4 bytes read per
    # sample, 4 written per trace
    for _ in range(3):
        sim.dvdt_peaks(score_dt)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record(stream)
    for _ in range(reps):
        sim.dvdt_peaks(score_dt)
    e1.record(stream)
    torch.cuda.synchronize()
    score_ms = e0.elapsed_time(e1) / reps
    score_bytes = len(grid) * (sim.n_samples + 1) * 4
    peak, peak_kind = hbm_peak()
    # end to end through the public call, host grid -> host score map
    e2e_s = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scores, _ = explore.explore(m, mapping, base)
        torch.cuda.synchronize()
        e2e_s.append(time.perf_counter() - t0)
    e2e_best = min(e2e_s)
    h2d = len(grid) * m.cell.n_params() * m.cell.n_sections * 4 + nt * 8
    if rank == 0:
        print(json.dumps({
            "metric": "compartment-steps/s (reference exploration run, TTPC 512 x 10000)", "value": rate,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": rate / EXPLORE_BASELINE, "dtype": "f32",
            "data": "the reference's shipped model and stimulus, its exploration grid",
            "config": {"workload": "explore", "model": "tests/golden/ttpc512 (BBP TTPC, 512 compartments)",
                       "n_sets": len(grid), "grid": "the reference's gen_params: GA parameter 0 (g_pas, every "
                       "section) over linspace(0, 10, 100) x parameter 2 (somatic gNaTs2_t) over "
                       "linspace(0, 20, 100)", "timesteps_per_step": nt,
                       "dt_ms": float(m.dts[0]), "launch_chunk": chunk,
                       "score": "scipy.signal.find_peaks(diff(v)/0.1, 15, distance=5) count per trace, on the GPU",
                       "l2": "state larger than L2 (no flush)"},
            "baseline": {"value": EXPLORE_BASELINE, "source": "GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/Data/"
                         "RunTimes.csv: 10000 sets, 42307.5 ms, the reference's GPU (not recorded)"},
            "e2e": {"value": cs_step / e2e_best, "unit": UNIT, "seconds": e2e_best, "seconds_each": e2e_s,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": len(grid) * 4,
                    "vs_baseline": cs_step / e2e_best / EXPLORE_BASELINE,
                    "includes": "grid and AllParams rows on the host, simulator creation, parameter upload, "
                                "init, run, score, score map to the host"},
            "score_kernel": {"ms": score_ms, "algorithmic_bytes": score_bytes,
                             "achieved_gbs": score_bytes / score_ms / 1e6, "peak_gbs": peak,
                             "frac": score_bytes / score_ms / 1e6 / peak, "peak_source": peak_kind,
                             "note": "k_dvdt_peaks over the run's trace buffer in place; traces in L2 "
                                     "after the first pass (127 MB, about L2's size)"},
            "scores": {"spiking_sets": int((c > 0).sum()), "max_count": int(c.max()),
                       "map_equals_e2e_call": bool(np.array_equal(scores.reshape(-1), c[:, 0]))},
            "gpu_launches": launches, "clocks": clk, "non_finite_instances": bad}))


def run_ga(args):
    """Config-5 line: GA time-to-score, surrogate-screened vs plain, on one
    GPU.  The cell: the 500-node HH-type cell, 12 free parameters (8
    conductances, 4 rate constants), 3 step protocols of 500 ms at dt 0.025
    ms.  The surrogate (4-layer MLP, width 512, GELU; in = 12 parameters +
    protocol one-hot, out = the 20 features) is trained once for the cell on
    `--ga-train` simulations drawn over the whole search space -- independent
    of any target, so one training serves every fit of the cell -- with the
    project's BF16 tcgen05 kernels.  Then, for each of `--ga-fits` targets
    (seeded parameter vectors): the plain GA (population `--ga-pop`, every
    offspring simulated, `--ga-gens` generations, every step on the device)
    sets the target score, its final best; the screened GA (the network
    ranks the offspring, the top 10 % are simulated, the network checked and
    fine-tuned every generation, every step on the device) runs until it
    reaches that score or until the plain GA's wall time has passed.
    value = the median over the fits of (screened time to the plain GA's
    final best score) / (plain GA wall time); null if a fit did not reach
    it.  The training cost is reported beside it, with the number of fits
    after which it has paid for itself."""
    import torch
    from neurogpu_b200 import ga
    torch.cuda.set_device(0)
    cell_prob = ga.FitProblem()
    fit = ga.train_surrogate(cell_prob, n_train=args.ga_train, epochs=args.ga_epochs, seed=0)
    fits = []
    for k in range(args.ga_fits):
        tu = np.random.default_rng(100 + k).uniform(-0.8, 0.8, cell_prob.n_params)
        prob = ga.FitProblem(target_u=tu)
        plain = ga.run_device(prob, args.ga_pop, args.ga_gens, seed=k + 1)
        sims_plain = prob.sim_count
        prob.sim_count = 0
        target = plain.best[-1]
        scr = ga.run_screened_device(prob, fit.net, args.ga_pop, 10 * args.ga_gens, seed=k + 1, target=target,
                                     time_budget=plain.time[-1])
        t_scr = scr.time_to(target)
        fits.append({
            "target_u": [round(float(x), 4) for x in tu],
            "plain": {"final_best": target, "seconds": plain.time[-1], "simulations": sims_plain,
                      "best_per_generation": plain.best, "time_per_generation": plain.time},
            "screened": {"final_best": scr.best[-1], "seconds": scr.time[-1], "generations": len(scr.best),
                         "simulations": prob.sim_count, "best_per_generation": scr.best,
                         "time_per_generation": scr.time, "time_to_plain_final_best": t_scr,
                         "surrogate_error_per_generation": [(g, round(e, 4), m) for g, e, m in scr.notes]},
            "time_ratio": None if t_scr is None else t_scr / plain.time[-1]})
    ratios = [f["time_ratio"] for f in fits]
    value = None if any(r is None for r in ratios) else float(np.median(ratios))
    saved = [f["plain"]["seconds"] - (f["screened"]["time_to_plain_final_best"] or f["plain"]["seconds"])
             for f in fits]
    train_s = fit.sim_seconds + fit.train_seconds
    print(json.dumps({
        "metric": "GA time-to-score ratio (surrogate-screened / plain)", "value": value, "unit": "ratio",
        "higher_is_better": False, "n_gpus": 1, "steps": len(fits), "warmup": 0,
        "dtype": "f32 sim, bf16 net", "data": "synthetic (seeded)", "vs_baseline": None,
        "config": {"workload": "ga", "population": args.ga_pop, "plain_generations": args.ga_gens,
                   "model": "hh 500 compartments, 12 parameters, 3 protocols x 500 ms", "screen_keep": 0.1,
                   "fits": args.ga_fits, "target": "each fit's plain GA final best score",
                   "surrogate_training_simulations": args.ga_train},
        "surrogate_training": {"simulations": fit.n_train, "simulation_seconds": fit.sim_seconds,
                               "training_seconds": fit.train_seconds, "epochs": args.ga_epochs,
                               "final_loss": fit.final_loss,
                               "fits_to_pay_back": None if min(saved) <= 0 else train_s / float(np.mean(saved))},
        "time_ratio_per_fit": ratios, "fits": fits}), flush=True)
    return 0


def run_ga_ops(args):
    """One JSON line of the device GA steps (csrc/ga.cuh) at the reference's
    GA size: bluepyopt's offspring_size 5000 (mu + lambda = 10,000), 12
    genes, 60 objectives (3 protocols x 20 features); NSGA-II also at 2,048
    and 32,768, and with 2 objectives (many fronts).  Device time with CUDA
    events on the current stream over `--steps` calls after `--warmup`; the
    numpy restatement (oracle/ga_numpy.py) on the host beside it where it
    finishes in seconds.  value = the NSGA-II selection at 10,000 x 60 (ms)."""
    import torch
    sys.path.insert(0, str(ROOT / "oracle"))
    import ga_numpy
    from neurogpu_b200.ga_device import DeviceGA, select_nsga2, select_truncation

    def dev_ms(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    def host_ms(fn, n=3):
        t = time.perf_counter()
        for _ in range(n):
            fn()
        return (time.perf_counter() - t) / n * 1e3

    rng = np.random.default_rng(0)
    mu, lam, genes = 5000, 5000, 12
    pop = rng.uniform(-1, 1, (mu, genes))
    rank = np.zeros(mu, np.int32)
    crowd = rng.normal(size=mu)
    ga = DeviceGA(genes, eta_c=20.0, eta_m=20.0, cx_prob=0.7, p_mut=0.3, seed=1)
    tp, tr, tc = (torch.tensor(x, device="cuda") for x in (pop, rank, crowd))
    out = {"offspring_5000x12": {"gpu_ms": dev_ms(lambda: ga.offspring(tp, tr, tc, lam, 3)),
                                 "numpy_ms": host_ms(lambda: ga_numpy.offspring(pop, rank, crowd, lam, -1.0, 1.0,
                                                                                20.0, 20.0, 0.7, 0.3, 1, 3))}}
    sc = rng.normal(size=mu + lam)
    ts = torch.tensor(sc, device="cuda")
    out["truncation_10000"] = {"gpu_ms": dev_ms(lambda: select_truncation(ts, mu)),
                               "numpy_ms": host_ms(lambda: ga_numpy.select_truncation(sc, mu))}
    for n, m in ((2048, 60), (10000, 60), (32768, 60), (10000, 2)):
        obj = rng.uniform(0, 1, (n, m))
        to = torch.tensor(obj, device="cuda")
        row = {"gpu_ms": dev_ms(lambda: select_nsga2(to, n // 2)), "fronts": int(select_nsga2(to, n // 2)[3])}
        if n <= 2048:
            row["numpy_ms"] = host_ms(lambda: ga_numpy.select_nsga2(obj, n // 2), 1)
        out[f"nsga2_{n}x{m}"] = row
    print(json.dumps({
        "metric": "NSGA-II selection time (10,000 x 60 objectives)", "value": out["nsga2_10000x60"]["gpu_ms"],
        "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "dtype": "f64", "data": "synthetic (seeded uniform objectives)", "vs_baseline": None,
        "config": {"workload": "ga_ops", "mu": mu, "lambda": lam, "genes": genes, "objectives": 60},
        "steps_ms": out}))


def run_gemm(args):
    """The surrogate network's hand-written tcgen05 BF16 GEMM (ngpu_gemm_bf16_tn,
    FP32 accumulation in tensor memory) at the network's training shapes
    (batch 8192, width 512: forward layers, the weight gradients over the
    batch) and at square sizes, against torch.matmul (cuBLAS) on the same
    operands.  Device time with CUDA events over `--steps` calls after
    `--warmup`, and per call inside a CUDA graph of 20 calls (graph_ms: the
    host's per-call work, which bounds the small shapes from Python, left
    out); value = TFLOP/s of the 8192^3 GEMM, frac of the measured cuBLAS
    bf16 peak (MEASURED_PEAKS.json bf16_tflops, burst)."""
    import torch
    from neurogpu_b200 import _ffi
    L = _ffi.lib()
    try:
        peak = float(json.loads(PEAKS_FILE.read_text())["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        peak, peak_kind = 1590.0, "fallback"

    def dev_ms(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    def graph_ms(fn, n=20):
        """Device time of one call with the host out of the loop: n calls
        captured once as a CUDA graph, the graph replayed after warm-up."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn()
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(n):
                fn()
        for _ in range(max(args.warmup, 1)):
            graph.replay()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        graph.replay()
        b.record()
        torch.cuda.synchronize()
        del graph
        return a.elapsed_time(b) / n

    rows = {}
    g = torch.Generator(device="cuda").manual_seed(0)
    # (name, M, N, K, bn, epilogue): epilogue 0 store fp32, 1 bias + GELU (three outputs),
    # 4 store fp32 with K split over CTAs
    shapes = [("fwd_hidden_8192x512x512", 8192, 512, 512, 128, 1),
              ("fwd_hidden_8192x512x512_bn256", 8192, 512, 512, 256, 1),
              ("fwd_input_8192x512x64", 8192, 512, 64, 128, 1), ("fwd_input_8192x512x64_bn256", 8192, 512, 64, 256, 1),
              ("fwd_out_8192x32x512", 8192, 32, 512, 32, 0), ("dW_512x512x8192", 512, 512, 8192, 128, 0),
              ("dW_512x512x8192_splitK", 512, 512, 8192, 128, 4),
              ("square_4096", 4096, 4096, 4096, 256, 0), ("square_8192", 8192, 8192, 8192, 256, 0)]
    for name, M, N, K, bn, epi in shapes:
        A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
        out = torch.empty(M, N, device="cuda", dtype=torch.float32)
        ob = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
        obt = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
        bias = torch.zeros(N, device="cuda", dtype=torch.float32)
        def ours():
            _ffi.check("ngpu_gemm_bf16_tn", L.ngpu_gemm_bf16_tn(
                A.data_ptr(), B.data_ptr(), M, N, K, K, K, epi, bn, out.data_ptr(),
                ob.data_ptr() if epi == 1 else None, obt.data_ptr() if epi == 1 else None, N, M,
                bias.data_ptr() if epi == 1 else None, None, torch.cuda.current_stream().cuda_stream))
        ms = dev_ms(ours)
        try:
            ms_graph = graph_ms(ours)
        except Exception as exc:  # capture refused: report the eager figure only
            print(f"gemm {name}: graph timing skipped ({exc})", file=sys.stderr)
            ms_graph = None
        ref = torch.matmul(A.float(), B.float().t()) if M * N * K <= 4096 ** 3 else None
        ours()
        torch.cuda.synchronize()
        err = None
        if ref is not None:
            got = out if epi == 0 else out - bias
            err = float((got - ref).abs().max() / ref.abs().max())
        ms_cublas = dev_ms(lambda: torch.matmul(A, B.t()))
        cb_out = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
        ms_cublas_graph = graph_ms(lambda: torch.matmul(A, B.t(), out=cb_out))
        fl = 2.0 * M * N * K
        rows[name] = {"ms": ms, "tflops": fl / ms / 1e9, "cublas_ms": ms_cublas,
                      "cublas_tflops": fl / ms_cublas / 1e9,
                      "graph_ms": ms_graph, "graph_tflops": fl / ms_graph / 1e9 if ms_graph else None,
                      "cublas_graph_ms": ms_cublas_graph, "bn": bn,
                      "epilogue": {0: "store f32", 1: "bias+gelu (f32, bf16, bf16^T)", 4: "store f32, split K"}[epi],
                      "max_rel_err_vs_fp32": err}
        del A, B, out, ob, obt, cb_out
    v = rows["square_8192"]["tflops"]
    print(json.dumps({
        "metric": "tcgen05 BF16 GEMM TFLOP/s (8192^3)", "value": v, "unit": "TFLOP/s", "higher_is_better": True,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "dtype": "bf16 (fp32 accumulate)",
        "data": "synthetic (seeded normal)", "vs_baseline": None,
        "config": {"workload": "gemm", "surrogate": "MLP width 512, batch 8192"},
        "roofline": {"bound": "tensor", "achieved": v, "peak": peak, "unit": "TFLOP/s", "frac": v / peak,
                     "peak_source": peak_kind},
        "shapes": rows}), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ga":
        return run_ga(args)
    if args.workload == "ga_ops":
        return run_ga_ops(args)
    if args.workload == "uneven_batch":
        return run_uneven(args)
    if args.workload == "gemm":
        return run_gemm(args)
    if args.workload == "explore":
        return run_explore(args)
    import torch
    from neurogpu_b200 import _ffi
    from neurogpu_b200.sim import Model, Simulator, run
    rank, world, local = dist_setup(args.gpus)
    w = workload(args.n_sets, args.model)
    n_inst = w.n_sets * w.n_stim
    total_steps = (args.warmup + args.steps) * args.chunk
    if total_steps > w.nt:
        raise SystemExit(f"warmup+steps x chunk = {total_steps} exceeds the protocol ({w.nt} steps)")
    model = Model(w.cell)
    sim = Simulator(model, w.n_sets, w.n_stim, "fp32")
    sim.set_params(w.params)
    sim.set_stimulus(w.amps, w.dts, w.stim_node, w.stim_area)
    sim.set_recording(w.rec_nodes, 1)
    stream = torch.cuda.current_stream()
    sim.init(w.v_init, stream)
    t = 0
    for _ in range(args.warmup):
        sim.advance(t, args.chunk, stream)
        t += args.chunk
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    torch.cuda.synchronize()
    barrier(world)
    _ffi.lib().ngpu_launch_count(1)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launch_ms = []
    ev0.record(stream)
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.advance(t, args.chunk, stream)
        b.record(stream)
        launch_ms.append((a, b))
        t += args.chunk
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = int(_ffi.lib().ngpu_launch_count(0))
    barrier(world)
    clk = clocks.stop() if clocks else None
    per_launch_ms = float(np.mean([a.elapsed_time(b) for a, b in launch_ms]))
    n_bad = sim.n_bad()
    comp_steps_rank = w.cell.n_nodes * args.chunk * n_inst * args.steps
    value, el_s = weak_scaling_rate(comp_steps_rank, ev0.elapsed_time(ev1) / 1e3, world)
    el_ms = el_s * 1e3

    # roofline of the advance kernel: bytes per launch / launch time.  The
    # bytes are the algorithmic B_c per compartment-step, or the DRAM bytes
    # ncu measured where fewer reach DRAM (parameter rows shared by many
    # nodes are read from L2): only bytes that move are credited.
    peak, peak_kind = hbm_peak()
    bc = w.cell.algorithmic_bytes_per_step() / w.cell.n_nodes
    tpcs = traffic_per_comp_step(args.model)
    bytes_cs = bc if tpcs is None else min(bc, tpcs)
    cs_launch = w.cell.n_nodes * n_inst * args.chunk
    achieved_gbs = bytes_cs * cs_launch / (per_launch_ms / 1e3) / 1e9
    achieved_alg_gbs = bc * cs_launch / (per_launch_ms / 1e3) / 1e9
    traffic = None if tpcs is None else tpcs * cs_launch

    # end to end through the public host-buffer entry point (ngpu_run)
    e2e = None
    if not args.no_e2e:
        we = w.subset(nt=args.e2e_steps)
        run(model, we.params, we.amps, we.dts, we.stim_node, we.stim_area, we.rec_nodes, we.v_init)
        torch.cuda.synchronize()
        samples = []
        for _ in range(5):  # the median of five calls: host-side work makes single calls noisy
            barrier(world)
            t0 = time.perf_counter()
            out = run(model, we.params, we.amps, we.dts, we.stim_node, we.stim_area, we.rec_nodes, we.v_init)
            samples.append(max_over_ranks(time.perf_counter() - t0, world))
        e2e_s = float(np.median(samples))
        h2d = we.params.nbytes + we.amps.nbytes + we.dts.nbytes + we.rec_nodes.nbytes
        e2e = {"value": we.compartment_steps() * world / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(out.nbytes),
               "timesteps": args.e2e_steps, "seconds": e2e_s, "calls_timed": len(samples),
               "seconds_each": samples}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.cpu_sample_sets // 1, args.cpu_sample_steps)

    if rank == 0:
        line = {
            "metric": MODELS[args.model][0], "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": args.model, "n_nodes": w.cell.n_nodes, "n_sets": w.n_sets,
                       "n_stim": w.n_stim, "instances_per_gpu": n_inst, "dt_ms": w.dt,
                       "timesteps_per_step": args.chunk, "l2": "state larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": achieved_gbs / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_compartment_step": bytes_cs,
                         "bytes_basis": "algorithmic" if bytes_cs == bc else "dram (ncu), below algorithmic",
                         "algorithmic_bytes_per_compartment_step": bc,
                         "dram_bytes_per_compartment_step": tpcs,
                         "frac_algorithmic": achieved_alg_gbs / peak,
                         "launch_ms": per_launch_ms},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "non_finite_instances": n_bad,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    model.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
