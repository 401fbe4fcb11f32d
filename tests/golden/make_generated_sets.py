"""Mechanism sets generated by neurogpu_b200.nmodl from the reference's own
.mod files, stored for the GPU tests (tests/test_generated_sets.py), which
run where the reference tree is absent.

  ttpc.json    NeuroGPU_Base/scripts/template/*.mod (the 13 BBP TTPC
               mechanisms; celsius 34, ena 50, ek -85, as in
               GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cu)
  mainen.json  Figures/FigureS4_mainen/*.mod (na, kv, km, kca, ca, cad and
               the pas copies; celsius 37, ena 60, ek -90, the PARAMETERs
               the reference's CParsed/AllModels.cu compiles in as constants)

Each file holds the GeneratedMechSet fields: the generator's CUDA source and
the set's layout (mechanisms, parameters, state rows, costs).  The CPU test
regenerates them where the reference tree is present and checks they are
unchanged.

Run: python tests/golden/make_generated_sets.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
from oracle_py import REFERENCE_DIR  # noqa: E402

OUT = HERE / "generated_sets"
TTPC_MODS = REFERENCE_DIR / "NeuroGPU_Base" / "scripts" / "template"
MAINEN_MODS = REFERENCE_DIR / "Figures" / "FigureS4_mainen"
# the PARAMETERs of the Mainen .mod files that the reference's generated
# channel code compiles in (Figures/FigureS4_mainen/CParsed/AllModels.cu)
MAINEN_CONSTANTS = {
    "ca": {"cao": 2.5, "vshift": 0, "temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "na": {"vshift": -5, "temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "kca": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "km": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "kv": {"temp": 23, "q10": 2.3, "vmin": -120, "vmax": 100},
    "cad": {"depth": 0.09334562733124982, "taur": 200.0, "cainf": 1e-4},
}
FIELDS = ("name", "mechs", "params", "mech_params", "state_rows", "param_defaults", "celsius", "source", "cost")


def generate(which: str):
    from neurogpu_b200 import nmodl
    if which == "ttpc":
        return nmodl.generate_from_files(sorted(p for p in TTPC_MODS.glob("*.mod") if p.stem != "branching"),
                                         name="ttpc_generated", celsius=34.0, reversal={"na": 50.0, "k": -85.0})
    return nmodl.generate_from_files(sorted(p for p in MAINEN_MODS.glob("*.mod") if p.stem != "branching"),
                                     name="mainen_generated", celsius=37.0, reversal={"na": 60.0, "k": -90.0},
                                     constants=MAINEN_CONSTANTS)


def to_json(g) -> str:
    d = {k: getattr(g, k) for k in FIELDS}
    return json.dumps(d, indent=1, sort_keys=True) + "\n"


def load(which: str):
    """The stored set as a GeneratedMechSet (not yet registered)."""
    from neurogpu_b200.nmodl import GeneratedMechSet
    d = json.loads((OUT / f"{which}.json").read_text())
    for k in ("mechs", "params", "state_rows", "param_defaults", "cost"):
        d[k] = tuple(d[k])
    d["mech_params"] = tuple(tuple(x) for x in d["mech_params"])
    return GeneratedMechSet(**d)


def main():
    OUT.mkdir(exist_ok=True)
    for which in ("ttpc", "mainen"):
        (OUT / f"{which}.json").write_text(to_json(generate(which)))
        print(which, "written")


if __name__ == "__main__":
    main()
