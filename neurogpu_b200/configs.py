"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset is involved: morphologies, parameter sets and stimuli are drawn
from ``numpy.random.default_rng(seed)`` with the sizes and distributions the
configurations name.

* ``passive_cable``  -- random binary tree of 128 compartments (20 um long,
  diameter U[1,4] um, Ra 100 Ohm cm, cm 1 uF/cm2, g_pas 1e-4 S/cm2,
  e_pas -70 mV); 32 instances with g_pas x U[0.5,2]; 0.5 nA soma step
  10-90 ms; dt 0.025 ms; 100 ms.
* ``hh_active``      -- 500-compartment tree (soma + 2 dendritic subtrees +
  axon) with the Mainen channel set (na m3h, kv, km, kca + cad, ca, pas);
  1024 instances x 8 conductances log-U[0.5,2] x nominal; 3 steps
  (0.2/0.5/1.0 nA); 500 ms at dt 0.025 ms.
* ``ttpc_like``      -- ~1500-compartment thick-tufted pyramidal morphology
  (soma, axon initial segment, basal trees, apical trunk with obliques and
  tuft) with the TTPC channel set (13 mechanisms); 4096 instances x 12
  conductances log-U[0.1,10] x nominal; 3 protocols; 2000 ms at dt 0.025 ms.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mechsets import MAINEN, TTPC, MechSet
from .model import CellModel, SectionSpec, build_model, cable_coefficients, random_binary_cable, \
    random_subtree


@dataclass
class Workload:
    name: str
    cell: CellModel
    params: np.ndarray        # float32 [n_sets, n_params, n_sections]
    amps: np.ndarray          # float32 [n_stim, nt] nA
    dt: float
    stim_node: int
    stim_area: float          # um2
    rec_nodes: np.ndarray     # int32
    v_init: float
    free: np.ndarray | None = None   # [n_sets, n_free] conductance multipliers
    seed: int = 0
    info: dict = field(default_factory=dict)

    def __post_init__(self):
        # the C ABI (and the reference's Stim_meta.csv reader) carries the area as float32
        self.stim_area = float(np.float32(self.stim_area))

    @property
    def n_sets(self) -> int:
        return int(self.params.shape[0])

    @property
    def n_stim(self) -> int:
        return int(self.amps.shape[0])

    @property
    def nt(self) -> int:
        return int(self.amps.shape[1])

    @property
    def dts(self) -> np.ndarray:
        return np.full(self.nt, self.dt, dtype=np.float32)

    def compartment_steps(self) -> int:
        return self.cell.n_nodes * self.nt * self.n_sets * self.n_stim

    def subset(self, n_sets: int | None = None, n_stim: int | None = None,
               nt: int | None = None) -> "Workload":
        ns = self.n_sets if n_sets is None else min(n_sets, self.n_sets)
        nst = self.n_stim if n_stim is None else min(n_stim, self.n_stim)
        ntt = self.nt if nt is None else min(nt, self.nt)
        return Workload(self.name, self.cell, np.ascontiguousarray(self.params[:ns]),
                        np.ascontiguousarray(self.amps[:nst, :ntt]), self.dt, self.stim_node,
                        self.stim_area, self.rec_nodes, self.v_init,
                        None if self.free is None else self.free[:ns], self.seed, dict(self.info))

    def take(self, sets) -> "Workload":
        """The workload restricted to the parameter sets `sets` (indices into
        this workload's sets, in the given order), every protocol, every step."""
        idx = np.asarray(sets, dtype=np.int64).reshape(-1)
        return Workload(self.name, self.cell, np.ascontiguousarray(self.params[idx]),
                        self.amps, self.dt, self.stim_node, self.stim_area, self.rec_nodes, self.v_init,
                        None if self.free is None else self.free[idx], self.seed, dict(self.info))


def step_amps(levels, nt: int, dt: float, t_on: float, t_off: float) -> np.ndarray:
    t = np.arange(nt) * dt
    on = (t >= t_on) & (t < t_off)
    return np.stack([np.where(on, lv, 0.0) for lv in levels]).astype(np.float32)


# ----------------------------------------------------------------------- 1
def passive_cable(n_sets: int = 32, t_stop: float = 100.0, dt: float = 0.025,
                  n_comp: int = 128, seed: int = 1) -> Workload:
    rng = np.random.default_rng(seed)
    parent, length, diam = random_binary_cable(rng, n_comp, 20.0, (1.0, 4.0))
    a, b, area = cable_coefficients(parent, length, diam, 100.0)
    n = parent.shape[0]
    mask = np.zeros((TTPC.n_mech, n), dtype=np.uint8)
    mask[TTPC.mech_index("pas")] = 1
    cell = CellModel(parent=parent, a=a, b=b, cm=np.ones(n), section=np.arange(n, dtype=np.int32),
                     n_sections=n, mechset=TTPC, mech_mask=mask, area=area,
                     region=np.zeros(n, dtype=np.int32), region_names=("cable",),
                     meta={"length_um": length, "diam_um": diam})
    cell.validate()
    scale = rng.uniform(0.5, 2.0, n_sets)
    params = np.zeros((n_sets, TTPC.n_params, n), dtype=np.float32)
    params[:, TTPC.param_index("g_pas"), :] = (1e-4 * scale)[:, None]
    params[:, TTPC.param_index("e_pas"), :] = -70.0
    nt = int(round(t_stop / dt))
    amps = step_amps([0.5], nt, dt, 10.0, 90.0)
    return Workload("passive_cable", cell, params, amps, dt, 0, float(area[0]),
                    np.array([0], dtype=np.int32), -70.0, scale[:, None], seed)


# ----------------------------------------------------------------------- 2
MAINEN_REGIONS = ("soma", "dend", "axon")
MAINEN_MECHS = {
    "soma": ("ca", "cad", "kca", "km", "kv", "na", "pas"),
    "dend": ("ca", "cad", "kca", "km", "na", "pas"),
    "axon": ("na", "kv", "pas"),
}
# nominal conductances (pS/um2) per region, Figures/FigureS4_mainen/myMainen.hoc:124-148
MAINEN_NOMINAL = {
    "soma": {"gbar_na": 20.0, "gbar_kv": 200.0, "gbar_km": 0.1, "gbar_kca": 3.0, "gbar_ca": 0.3},
    "dend": {"gbar_na": 20.0, "gbar_km": 0.1, "gbar_kca": 3.0, "gbar_ca": 0.3},
    "axon": {"gbar_na": 30000.0, "gbar_kv": 2000.0},
}
# kinetic constants, Figures/FigureS4_mainen/*.mod PARAMETER blocks
MAINEN_FIXED = {
    "cao_ca": 2.5, "caix_kca": 1.0, "Ra_kca": 0.01, "Rb_kca": 0.02,
    "tha_km": -30.0, "qa_km": 9.0, "Ra_km": 0.001, "Rb_km": 0.001,
    "tha_kv": 25.0, "qa_kv": 9.0, "Ra_kv": 0.02, "Rb_kv": 0.002,
    "tha_na": -35.0, "qa_na": 9.0, "Ra_na": 0.182, "Rb_na": 0.124, "thi1_na": -50.0,
    "thi2_na": -75.0, "qi_na": 5.0, "thinf_na": -65.0, "qinf_na": 6.2, "Rg_na": 0.0091,
    "Rd_na": 0.024, "g_pas": 3.3e-5, "e_pas": -70.0,
}
# the 8 free conductances: (parameter, regions)
MAINEN_FREE = (("gbar_na", ("soma", "dend")), ("gbar_na", ("axon",)), ("gbar_kv", ("soma",)),
               ("gbar_kv", ("axon",)), ("gbar_km", ("soma", "dend")), ("gbar_kca", ("soma", "dend")),
               ("gbar_ca", ("soma", "dend")), ("g_pas", ("soma", "dend", "axon")))


def hh_morphology(rng: np.random.Generator, n_target: int = 500) -> list[SectionSpec]:
    secs = [SectionSpec(-1, 1, 20.0, 20.0, 0)]
    secs.append(SectionSpec(0, 5, 4.0, 3.0, 2))      # hillock
    secs.append(SectionSpec(1, 15, 2.0, 1.5, 2))     # initial segment
    secs.append(SectionSpec(2, 30, 10.0, 1.0, 2))    # axon
    rest = n_target - 51
    half = rest // 2
    random_subtree(rng, 0, half, 1, 15.0, 2.5, 0.8, (4, 10), secs)
    random_subtree(rng, 0, rest - half, 1, 15.0, 2.5, 0.8, (4, 10), secs)
    return secs


def _region_params(cell: CellModel, mechset: MechSet, nominal: dict, fixed: dict,
                   gradient=None) -> np.ndarray:
    base = np.zeros((mechset.n_params, cell.n_sections), dtype=np.float64)
    for s in range(cell.n_sections):
        rname = cell.region_names[cell.region[s]]
        for k, v in fixed.items():
            base[mechset.param_index(k), s] = v
        for k, v in nominal.get(rname, {}).items():
            base[mechset.param_index(k), s] = v
        if gradient is not None:
            gradient(base, s, rname)
    return base


def _apply_free(cell: CellModel, mechset: MechSet, base: np.ndarray, free_spec, mult: np.ndarray) -> np.ndarray:
    n_sets = mult.shape[0]
    params = np.broadcast_to(base, (n_sets,) + base.shape).copy()
    sec_region = np.array([cell.region_names[r] for r in cell.region])
    for j, (pname, regions) in enumerate(free_spec):
        cols = np.nonzero(np.isin(sec_region, regions))[0]
        pi = mechset.param_index(pname)
        params[:, pi, cols] *= mult[:, j:j + 1]
    return params.astype(np.float32)


def hh_active(n_sets: int = 1024, t_stop: float = 500.0, dt: float = 0.025, n_comp: int = 500,
              seed: int = 2, levels=(0.2, 0.5, 1.0)) -> Workload:
    rng = np.random.default_rng(seed)
    secs = hh_morphology(rng, n_comp)
    cell = build_model(secs, MAINEN, MAINEN_REGIONS, MAINEN_MECHS, ra=150.0,
                       cm_of_region={"soma": 0.75, "dend": 1.5, "axon": 0.75})
    base = _region_params(cell, MAINEN, MAINEN_NOMINAL, MAINEN_FIXED)
    mult = np.exp(rng.uniform(np.log(0.5), np.log(2.0), (n_sets, len(MAINEN_FREE))))
    params = _apply_free(cell, MAINEN, base, MAINEN_FREE, mult)
    nt = int(round(t_stop / dt))
    amps = step_amps(levels, nt, dt, 50.0, 450.0)
    return Workload("hh_active", cell, params, amps, dt, 0, float(cell.area[0]),
                    np.array([0], dtype=np.int32), -70.0, mult, seed)


def uneven_batch(n_sets: int = 8192, sizes=(200, 800, 1500, 3000), t_stop: float = 500.0, dt: float = 0.025,
                 seed: int = 4, levels=(0.1, 0.2, 0.4, 0.7, 1.0)) -> list[Workload]:
    """An uneven batch: seeded HH-type trees of the given compartment counts
    (the hh_active channel set and parameter sampling), n_sets split evenly
    over them, five step protocols shared by all (one instance = one set x
    one protocol)."""
    per = n_sets // len(sizes)
    out = []
    for k, n in enumerate(sizes):
        w = hh_active(n_sets=per, t_stop=t_stop, dt=dt, n_comp=n, seed=seed * 100 + k, levels=levels)
        w.name = f"uneven_{n}"
        out.append(w)
    return out


# ----------------------------------------------------------------------- 3
TTPC_REGIONS = ("soma", "axon", "basal", "trunk", "oblique", "tuft")
TTPC_MECHS = {
    "soma": ("Ca_HVA", "Ca_LVAst", "CaDynamics_E2", "Ih", "K_Pst", "K_Tst", "NaTs2_t", "pas",
             "SK_E2", "SKv3_1"),
    "axon": ("Ca_HVA", "Ca_LVAst", "CaDynamics_E2", "K_Pst", "K_Tst", "Nap_Et2", "NaTa_t", "pas",
             "SK_E2", "SKv3_1"),
    "basal": ("Ih", "pas"),
    "trunk": ("Ih", "Im", "NaTs2_t", "pas", "SKv3_1"),
    "oblique": ("Ih", "Im", "NaTs2_t", "pas", "SKv3_1"),
    "tuft": ("Ca_HVA", "Ca_LVAst", "CaDynamics_E2", "Ih", "Im", "NaTs2_t", "pas", "SK_E2", "SKv3_1"),
}
# nominal values of the BBP L5 TTPC model; somatic/axonal values as in the
# reference's GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/Data/AllParams_reference.csv
TTPC_NOMINAL = {
    "soma": {"gCa_HVAbar_Ca_HVA": 0.000994, "gCa_LVAstbar_Ca_LVAst": 0.000333,
             "gamma_CaDynamics_E2": 0.000609, "decay_CaDynamics_E2": 210.485,
             "gNaTs2_tbar_NaTs2_t": 0.983955, "gSK_E2bar_SK_E2": 0.008407,
             "gSKv3_1bar_SKv3_1": 0.303472, "gK_Pstbar_K_Pst": 0.0, "gK_Tstbar_K_Tst": 0.0},
    "axon": {"gCa_HVAbar_Ca_HVA": 0.00099, "gCa_LVAstbar_Ca_LVAst": 0.008752,
             "gamma_CaDynamics_E2": 0.00291, "decay_CaDynamics_E2": 287.199,
             "gK_Pstbar_K_Pst": 0.973538, "gK_Tstbar_K_Tst": 0.089259,
             "gNap_Et2bar_Nap_Et2": 0.006827, "gNaTa_tbar_NaTa_t": 3.137968,
             "gSK_E2bar_SK_E2": 0.007104, "gSKv3_1bar_SKv3_1": 1.021945},
    "basal": {},
    "trunk": {"gNaTs2_tbar_NaTs2_t": 0.026145, "gSKv3_1bar_SKv3_1": 0.004226, "gImbar_Im": 0.000143},
    "oblique": {"gNaTs2_tbar_NaTs2_t": 0.026145, "gSKv3_1bar_SKv3_1": 0.004226, "gImbar_Im": 0.000143},
    "tuft": {"gNaTs2_tbar_NaTs2_t": 0.026145, "gSKv3_1bar_SKv3_1": 0.004226, "gImbar_Im": 0.000143,
             "gCa_HVAbar_Ca_HVA": 5.55e-5, "gCa_LVAstbar_Ca_LVAst": 0.00187,
             "gamma_CaDynamics_E2": 0.0005, "decay_CaDynamics_E2": 80.0, "gSK_E2bar_SK_E2": 0.0012},
}
TTPC_FIXED = {"depth_CaDynamics_E2": 0.1, "minCai_CaDynamics_E2": 1e-4, "ehcn_Ih": -45.0,
              "g_pas": 3e-5, "e_pas": -75.0, "zTau_SK_E2": 1.0, "gIhbar_Ih": 8e-5}
TTPC_FREE = (("gNaTs2_tbar_NaTs2_t", ("soma",)), ("gNaTa_tbar_NaTa_t", ("axon",)),
             ("gNap_Et2bar_Nap_Et2", ("axon",)), ("gK_Pstbar_K_Pst", ("axon",)),
             ("gK_Tstbar_K_Tst", ("axon",)), ("gSKv3_1bar_SKv3_1", ("soma",)),
             ("gSKv3_1bar_SKv3_1", ("axon",)), ("gSK_E2bar_SK_E2", ("soma", "axon")),
             ("gCa_HVAbar_Ca_HVA", ("soma",)), ("gCa_LVAstbar_Ca_LVAst", ("axon",)),
             ("gIhbar_Ih", TTPC_REGIONS), ("gImbar_Im", ("trunk", "oblique", "tuft")))


def ttpc_morphology(rng: np.random.Generator, n_basal_trees: int = 6, basal_each: int = 100,
                    trunk_secs: int = 30, trunk_nseg: int = 8, oblique_each: int = 12,
                    tuft: int = 240) -> list[SectionSpec]:
    secs = [SectionSpec(-1, 1, 20.0, 20.0, 0)]
    secs.append(SectionSpec(0, 30, 2.0, 1.2, 1))
    secs.append(SectionSpec(1, 30, 2.0, 1.0, 1))
    for _ in range(n_basal_trees):
        random_subtree(rng, 0, basal_each, 2, 10.0, 1.6, 0.8, (4, 10), secs)
    psec = 0
    for k in range(trunk_secs):
        d = 4.0 - 2.5 * k / max(1, trunk_secs - 1)
        secs.append(SectionSpec(psec, trunk_nseg, 10.0, d, 3))
        psec = len(secs) - 1
        random_subtree(rng, psec, oblique_each, 4, 10.0, 0.9, 0.85, (3, 6), secs)
    random_subtree(rng, psec, tuft, 5, 10.0, 1.5, 0.8, (4, 10), secs)
    return secs


def ttpc_like(n_sets: int = 4096, t_stop: float = 2000.0, dt: float = 0.025, seed: int = 3,
              levels=(0.3, 0.6, 0.9)) -> Workload:
    rng = np.random.default_rng(seed)
    secs = ttpc_morphology(rng)
    cell = build_model(secs, TTPC, TTPC_REGIONS, TTPC_MECHS, ra=100.0,
                       cm_of_region={"soma": 1.0, "axon": 1.0, "basal": 2.0, "trunk": 2.0,
                                     "oblique": 2.0, "tuft": 2.0})
    # section mid-point path distance from the soma, for the Ih gradient
    n = cell.n_nodes
    length = cell.meta["length_um"]
    dist = np.zeros(n)
    for i in range(1, n):
        dist[i] = dist[cell.parent[i]] + 0.5 * (length[i] + length[cell.parent[i]])
    sec_dist = np.zeros(cell.n_sections)
    cnt = np.zeros(cell.n_sections)
    np.add.at(sec_dist, cell.section, dist)
    np.add.at(cnt, cell.section, 1)
    sec_dist /= np.maximum(cnt, 1)
    ih = TTPC.param_index("gIhbar_Ih")

    def gradient(base, s, rname):
        if rname in ("trunk", "oblique", "tuft"):  # BBP exponential Ih distribution
            base[ih, s] = 8e-5 * (-0.8696 + 2.087 * np.exp(0.0031 * sec_dist[s]))

    base = _region_params(cell, TTPC, TTPC_NOMINAL, TTPC_FIXED, gradient)
    mult = np.exp(rng.uniform(np.log(0.1), np.log(10.0), (n_sets, len(TTPC_FREE))))
    params = _apply_free(cell, TTPC, base, TTPC_FREE, mult)
    nt = int(round(t_stop / dt))
    amps = step_amps(levels, nt, dt, 100.0, 1900.0)
    return Workload("ttpc_like", cell, params, amps, dt, 0, float(cell.area[0]),
                    np.array([0], dtype=np.int32), -65.0, mult, seed)


CONFIGS = {"passive_cable": passive_cable, "hh_active": hh_active, "ttpc_like": ttpc_like}
