#!/usr/bin/env python
"""Builds the committed golden fixtures of tests/golden/ from the reference
tree (run here, where the reference is mounted; the GPU box only reads the
results).

1. Copies the input files of three reference models (data, not code):
     ttpc512/   GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/Data/{BasicConstSegP.csv,
                Sim.csv, Stim_meta.csv, Stim_raw0.csv, times.csv,
                AllParams_reference.csv, AllParams_for_params.csv, opt_table.csv}
     mainen384/ Figures/FigureS4_mainen/Data/{BasicConstSegP.csv, ParamsM.csv,
                Sim.csv, Stim_meta.csv, Stim_raw.csv, times.csv} + Fmatrix.csv
     passive384/ Figures/FigureS3_passive/Data/{same} + Fmatrix.csv
3. Feeds a seeded set of number tokens (and every value of the shipped
   AllParams) to the reference's own AllParams parser (oracle/_ref/ref_atof)
   and stores tokens and resulting float32 bits in atof_vectors.npz.
2. Evaluates the reference's OWN channel functions (built from its sources by
   oracle/build_ref.sh into oracle/_ref/libref_{ttpc,mainen}.so) on a seeded
   grid of voltages / states / parameters, mechanism by mechanism, and stores
   inputs and outputs in channels_{ttpc,mainen}.npz.
"""
from __future__ import annotations

import ctypes as C
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
from oracle_py import REFERENCE_DIR as REF  # noqa: E402

MODELS = {
    "ttpc512": ("GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/Data",
                ["BasicConstSegP.csv", "Sim.csv", "Stim_meta.csv", "Stim_raw0.csv", "times.csv",
                 "AllParams_reference.csv", "AllParams_for_params.csv", "opt_table.csv"], None),
    "mainen384": ("Figures/FigureS4_mainen/Data",
                  ["BasicConstSegP.csv", "ParamsM.csv", "Sim.csv", "Stim_meta.csv", "Stim_raw.csv",
                   "times.csv"], "Figures/FigureS4_mainen/Fmatrix.csv"),
    "passive384": ("Figures/FigureS3_passive/Data",
                   ["BasicConstSegP.csv", "ParamsM.csv", "Sim.csv", "Stim_meta.csv", "Stim_raw.csv",
                    "times.csv"], "Figures/FigureS3_passive/Fmatrix.csv"),
}


def copy_models() -> None:
    for name, (sub, files, fmat) in MODELS.items():
        out = HERE / name
        out.mkdir(exist_ok=True)
        for f in files:
            shutil.copyfile(REF / sub / f, out / f)
        if fmat:
            shutil.copyfile(REF / fmat, out / "Fmatrix.csv")


def channel_vectors() -> None:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py
    for ms, name, n_states, n_params, n_mech, skip in (
            (oracle_py.MECHSET_TTPC, "ttpc", 19, 19, 13, ()),
            (oracle_py.MECHSET_MAINEN, "mainen", 8, 34, 9, (7, 8))):
        L = oracle_py.ref_channels(ms)
        if L is None:
            raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` first")
        fn = L.ref_ttpc_mech if ms == oracle_py.MECHSET_TTPC else L.ref_mainen_mech
        rng = np.random.default_rng(2024 + ms)
        recs = []
        for mech in range(n_mech):
            if mech in skip:
                continue
            for what in (0, 1, 2):
                for _ in range(64):
                    v = np.float32(rng.choice([rng.uniform(-110, 50), -27.0, -38.0, -66.0, -32.0, -60.0]))
                    dt = np.float32(rng.choice([0.025, 0.1]))
                    s = np.zeros(n_states + 3, dtype=np.float32)
                    s[:n_states] = rng.uniform(0, 1, n_states)
                    s[n_states] = rng.uniform(5e-5, 5e-3)       # cai
                    s[n_states + 1] = 130.0                      # eca
                    s[n_states + 2] = rng.uniform(-0.02, 0.0)    # ica
                    p = np.abs(rng.normal(0.5, 0.3, n_params)).astype(np.float32) + np.float32(0.05)
                    s_in = s.copy()
                    g = C.c_float()
                    I = fn(mech, what, dt, v, s.ctypes.data, p.ctypes.data, C.byref(g))
                    recs.append((mech, what, v, dt, s_in, p, s.copy(), I, g.value))
        np.savez_compressed(
            HERE / f"channels_{name}.npz",
            mech=np.array([r[0] for r in recs], dtype=np.int32),
            what=np.array([r[1] for r in recs], dtype=np.int32),
            v=np.array([r[2] for r in recs], dtype=np.float32),
            dt=np.array([r[3] for r in recs], dtype=np.float32),
            s_in=np.stack([r[4] for r in recs]), p=np.stack([r[5] for r in recs]),
            s_out=np.stack([r[6] for r in recs]), I=np.array([r[7] for r in recs]),
            G=np.array([r[8] for r in recs], dtype=np.float32))


def atof_vectors() -> None:
    import subprocess
    exe = ROOT / "oracle" / "_ref" / "ref_atof"
    if not exe.exists():
        raise SystemExit("oracle/_ref/ref_atof is not built: run oracle/build_ref.sh first")
    rng = np.random.default_rng(77)
    toks = []
    for _ in range(4000):
        x = float(np.float32(rng.choice([1, -1]) * 10 ** rng.uniform(-9, 4)))
        toks.append(str(rng.choice([f"{x:.5E}", f"{x:.5e}", f"{x:.9e}", f"{x:.3f}", f" {x:.6e}"])))
    toks += [t.strip() for t in (HERE / "ttpc512" / "AllParams_reference.csv").read_text().split(",")[1:]
             if t.strip()]
    out = subprocess.run([str(exe)], input="\n".join(toks) + "\n", capture_output=True, text=True,
                         check=True).stdout.split()
    bits = np.array([int(h, 16) for h in out], dtype=np.uint32)
    np.savez_compressed(HERE / "atof_vectors.npz", tokens=np.array(toks), bits=bits)


if __name__ == "__main__":
    copy_models()
    channel_vectors()
    atof_vectors()
    print("golden fixtures written to", HERE)
