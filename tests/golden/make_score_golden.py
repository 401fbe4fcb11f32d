#!/usr/bin/env python
"""Golden vectors for neurogpu_b200/score_functions.py from the reference's
own GUI/score_functions.py (pure numpy, imported from the reference tree; run
here, where the reference is mounted).

Traces: the FP64 oracle on the shipped 512-node TTPC model (tests/golden/
ttpc512), parameter sets from make_ref_traces.param_sets, soma voltage,
dt 0.1 ms, an 800-sample window (5-85 ms) holding the early burst (2-3
spikes per trace).  Pairs: the
first set is the target; data are the other sets, a flat trace at the
resting level (no spikes), the target itself (zero scores) and the target
shifted by 2 mV.  Writes score_vectors.npz: target, data [n, 800], names,
scores [n_functions, n].
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))
from oracle_py import REFERENCE_DIR  # noqa: E402

REF_SCORES = REFERENCE_DIR / "GUI" / "score_functions.py"

NAMES = ["chi_square_normal", "abs_cumsum_diff", "comp_rest_potential", "comp_width", "comp_width_avg",
         "comp_height", "comp_height_avg", "traj_score_1", "traj_score_2", "traj_score_3", "isi",
         "rev_dot_product", "KL_divergence", "traj_score_single_peak", "DTWDistance"]


def traces() -> tuple[np.ndarray, np.ndarray]:
    import make_ref_traces as M
    import oracle_py
    m = M.model_inputs()
    c = m.cell
    p = M.param_sets(6, 0.2, seed=77)
    v = oracle_py.run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask, p,
                      m.amps, m.dts, m.stim_node, m.stim_area, m.rec_nodes, m.v_init)[:, 0, 0]
    w = v[:, 50:850]
    target = w[0]
    data = [w[k] for k in range(1, w.shape[0])]
    data += [np.full(800, w[0, -1]), target.copy(), target + 2.0]
    return target, np.stack(data)


def main() -> None:
    spec = importlib.util.spec_from_file_location("ref_score_functions", REF_SCORES)
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    target, data = traces()
    scores = np.full((len(NAMES), data.shape[0]), np.nan)
    for i, name in enumerate(NAMES):
        f = getattr(ref, name)
        for j in range(data.shape[0]):
            try:
                scores[i, j] = float(f(list(target), list(data[j]), 0.1))
            except Exception:         # the reference raises on some inputs (kept as NaN)
                scores[i, j] = np.nan
    np.savez_compressed(HERE / "score_vectors.npz", target=target, data=data, names=np.array(NAMES),
                        scores=scores)
    print("wrote", HERE / "score_vectors.npz")


if __name__ == "__main__":
    main()
