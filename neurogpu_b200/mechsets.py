"""Mechanism sets compiled into libngpu, with the reference's names and order.

A mechanism set is the channel library of one model family.  The reference
generates one per model (``AllModels.cu``); its mechanism order is the
column order of ``boolModel`` (BasicConstSegP.csv line 9) and its parameter
order is the row order of every AllParams.csv parameter block:

* TTPC   -- GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cuh:10-23 and
  the call list at src/CudaStuff.cu:220 (13 mechanisms, 19 parameters).
* MAINEN -- Figures/FigureS4_mainen/CParsed/AllModels.cuh:10-23 and :63
  (9 mechanisms, 34 parameters).
"""
from __future__ import annotations

from dataclasses import dataclass

from ._ffi import MECHSET_MAINEN, MECHSET_TTPC


@dataclass(frozen=True)
class MechSet:
    id: int
    name: str
    mechs: tuple[str, ...]
    params: tuple[str, ...]
    # parameter indices read by each mechanism (same order as mechs)
    mech_params: tuple[tuple[int, ...], ...]
    celsius: float

    @property
    def n_mech(self) -> int:
        return len(self.mechs)

    @property
    def n_params(self) -> int:
        return len(self.params)

    def mech_index(self, name: str) -> int:
        return self.mechs.index(name)

    def param_index(self, name: str) -> int:
        return self.params.index(name)


TTPC = MechSet(
    id=MECHSET_TTPC,
    name="ttpc",
    mechs=("Ca_HVA", "Ca_LVAst", "CaDynamics_E2", "Ih", "Im", "K_Pst", "K_Tst", "Nap_Et2",
           "NaTa_t", "NaTs2_t", "pas", "SK_E2", "SKv3_1"),
    params=("gCa_HVAbar_Ca_HVA", "gCa_LVAstbar_Ca_LVAst", "gamma_CaDynamics_E2",
            "decay_CaDynamics_E2", "depth_CaDynamics_E2", "minCai_CaDynamics_E2", "gIhbar_Ih",
            "ehcn_Ih", "gImbar_Im", "gK_Pstbar_K_Pst", "gK_Tstbar_K_Tst", "gNap_Et2bar_Nap_Et2",
            "gNaTa_tbar_NaTa_t", "gNaTs2_tbar_NaTs2_t", "g_pas", "e_pas", "gSK_E2bar_SK_E2",
            "zTau_SK_E2", "gSKv3_1bar_SKv3_1"),
    mech_params=((0,), (1,), (2, 3, 4, 5), (6, 7), (8,), (9,), (10,), (11,), (12,), (13,),
                 (14, 15), (16, 17), (18,)),
    celsius=34.0,
)

MAINEN = MechSet(
    id=MECHSET_MAINEN,
    name="mainen",
    mechs=("ca", "cad", "kca", "km", "kv", "na", "pas", "pas2", "pasx"),
    params=("gbar_ca", "cao_ca", "gbar_kca", "caix_kca", "Ra_kca", "Rb_kca", "gbar_km", "tha_km",
            "qa_km", "Ra_km", "Rb_km", "gbar_kv", "tha_kv", "qa_kv", "Ra_kv", "Rb_kv", "gbar_na",
            "tha_na", "qa_na", "Ra_na", "Rb_na", "thi1_na", "thi2_na", "qi_na", "thinf_na",
            "qinf_na", "Rg_na", "Rd_na", "g_pas", "e_pas", "g_pas2", "e_pas2", "g_pasx", "e_pasx"),
    mech_params=((0, 1), (), (2, 3, 4, 5), (6, 7, 8, 9, 10), (11, 12, 13, 14, 15),
                 tuple(range(16, 28)), (28, 29), (30, 31), (32, 33)),
    celsius=37.0,
)

BY_ID = {TTPC.id: TTPC, MAINEN.id: MAINEN}
BY_NAME = {TTPC.name: TTPC, MAINEN.name: MAINEN}
