"""File-compatible replacement of the reference's neuroGPU binary.

The reference's GA driver runs ``../bin/neuroGPU <stim_ind>`` once per
stimulus (Figures/Figure4_DEAP/neurogpu_multistim_evaluator_par.py:175).  The
binary (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/kernel.cu:8-33,
MainC.cu:589-626, CudaStuff.cu:518-587):

* takes its GPU from argv[1] (0 without an argument);
* reads, relative to its working directory, ../Data/BasicConstSegP.csv,
  Sim.csv, Stim_meta.csv, times.csv, AllParams.csv and Stim_raw<dev>.csv
  (Stim_raw.csv without an argument; Util.cu:359-364);
* writes ../Data/VHotP<dev>.dat (int32 count, int32 3, float64 V
  [set][stim][rec][t]) and ../Data/RunTimes.csv ("NSets,ms").

This command does the same through libngpu, so the driver runs unchanged
with ``neurogpu_b200/bin/neuroGPU`` in place of the binary.  Differences:
recording sites are honoured at any node (the reference records node
RecSite % 32 correctly only for sites below 32, CudaStuff.cu:243-247); with
fewer GPUs than the index, device index % count is used and the files keep
the index the driver asked for; errors exit non-zero with a message (the
reference prints and exits 0).  ``--data`` overrides ../Data and
``--check`` reads and validates every input without touching a GPU.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

from . import formats


def _parse(argv):
    ap = argparse.ArgumentParser(prog="neuroGPU", description=__doc__.split("\n\n")[0])
    ap.add_argument("stim_ind", nargs="?", type=int, default=None,
                    help="GPU index and Stim_raw<index>.csv suffix (reference argv[1])")
    ap.add_argument("--data", default=None, help="Data directory (default: ../Data, as the reference)")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--check", action="store_true", help="read and validate the inputs only")
    return ap.parse_args(argv)


def main(argv=None) -> int:
    a = _parse(argv)
    data = Path(a.data) if a.data else Path.cwd().parent / "Data"
    idx = 0 if a.stim_ind is None else a.stim_ind
    if idx < 0:
        print("neuroGPU: the stimulus index must be >= 0", file=sys.stderr)
        return 2
    try:
        m = formats.read_data_dir(data, stim_index=a.stim_ind, params_file="AllParams.csv"
                                  if (data / "AllParams.csv").exists() else None)
    except (OSError, ValueError, IndexError) as e:
        print(f"neuroGPU: cannot read {data}: {e}", file=sys.stderr)
        return 1
    n_sets = m.params.shape[0]
    if a.check:
        print(f"neuroGPU: {data}: {m.cell.n_nodes} nodes, {n_sets} sets, {m.amps.shape[0]} stimuli x "
              f"{m.amps.shape[1]} steps, stimulus node {m.stim_node}, recording {list(m.rec_nodes)}")
        return 0
    import ctypes as C

    from . import _ffi
    from .sim import run
    try:
        L = _ffi.lib()
        n_dev = C.c_int32()
        _ffi.check("ngpu_device_count", L.ngpu_device_count(C.byref(n_dev)))
        if n_dev.value < 1:
            print("neuroGPU: no CUDA device", file=sys.stderr)
            return 1
        _ffi.check("ngpu_set_device", L.ngpu_set_device(idx % n_dev.value))
        t0 = time.perf_counter()
        out = run(m.cell, m.params, m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init,
                  precision=a.precision)
        ms = (time.perf_counter() - t0) * 1e3
    except (_ffi.NgpuError, OSError, RuntimeError) as e:
        print(f"neuroGPU: {e}", file=sys.stderr)
        return 1
    formats.write_vhot(data / f"VHotP{idx}.dat", out.astype(np.float64))
    formats.write_run_times(data / "RunTimes.csv", n_sets, ms)
    print(f"neuroGPU: {n_sets} sets x {m.amps.shape[0]} stimuli x {m.amps.shape[1]} steps in {ms:.1f} ms "
          f"-> {data / f'VHotP{idx}.dat'}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
