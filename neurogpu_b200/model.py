"""Cell models: tree topology, cable coefficients and channel placement.

A :class:`CellModel` holds exactly what the reference's BasicConstSegP.csv
carries for the hot path (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/MainC.cu:
335-551): a tree in Hines order, the two axial coupling coefficients of every
node, membrane capacitance, the node -> parameter-section map (SegToComp) and
the per-node mechanism mask (boolModel).  The level schedule the reference
also stores there (Fathers, RelVec, CompByLevel32, FIdxs, ...) is derived
data; :mod:`neurogpu_b200.formats` recomputes the parts that tests pin.

Coefficient convention (row i of the node matrix):
    d_i dV_i + a_i dV_parent(i) + sum_{c child of i} b_c dV_c = rhs_i
``a`` is the reference's ``f`` (Fmatrix.csv column A) and ``b`` its ``e``
(column B), both reversed into node order.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from .mechsets import BY_ID, MechSet


@dataclass
class CellModel:
    parent: np.ndarray          # int32 [N], -1 at the root, parent[i] < i
    a: np.ndarray               # float64 [N]
    b: np.ndarray               # float64 [N]
    cm: np.ndarray              # float64 [N] uF/cm2
    section: np.ndarray         # int32 [N] node -> section
    n_sections: int
    mechset: MechSet
    mech_mask: np.ndarray       # uint8 [n_mech, N]
    area: np.ndarray | None = None      # um2 per node (synthetic models)
    region: np.ndarray | None = None    # region label index per section
    region_names: tuple[str, ...] = ()
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.parent.shape[0])

    def validate(self) -> None:
        n = self.n_nodes
        p = self.parent
        if p.shape != (n,) or p[0] != -1:
            raise ValueError("parent[0] must be -1")
        if n > 1 and (np.any(p[1:] < 0) or np.any(p[1:] >= np.arange(1, n))):
            raise ValueError("tree is not in Hines order (parent < child)")
        for arr, nm in ((self.a, "a"), (self.b, "b"), (self.cm, "cm")):
            if arr.shape != (n,) or not np.all(np.isfinite(arr)):
                raise ValueError(f"{nm} must be finite with one value per node")
        if self.mech_mask.shape != (self.mechset.n_mech, n):
            raise ValueError("mech_mask must be [n_mech, n_nodes]")
        if self.section.min() < 0 or self.section.max() >= self.n_sections:
            raise ValueError("section index out of range")

    def children_counts(self) -> np.ndarray:
        return np.bincount(self.parent[1:], minlength=self.n_nodes)

    def depth(self) -> np.ndarray:
        d = np.zeros(self.n_nodes, dtype=np.int64)
        for i in range(1, self.n_nodes):
            d[i] = d[self.parent[i]] + 1
        return d

    def n_params(self) -> int:
        return self.mechset.n_params

    def algorithmic_bytes_per_step(self) -> int:
        """Sum over nodes of B_c = 8*(1+S_c) + 8 + 4*P_c (bytes per node-step).

        V read+write (8), Kahan term read+write (8), S_c channel state
        variables read+write (8 each, cai and the carried ica included), P_c
        FP32 parameters read (4 each)."""
        st_rows = getattr(self.mechset, "state_rows", None) or {
            "ttpc": (2, 2, 2, 1, 1, 2, 2, 2, 2, 2, 0, 1, 1),
            "mainen": (2, 2, 1, 1, 1, 2, 0, 0, 0)}[self.mechset.name]
        total = 0
        for i in range(self.n_nodes):
            on = np.nonzero(self.mech_mask[:, i])[0]
            S = sum(st_rows[k] for k in on)
            P = sum(len(self.mechset.mech_params[k]) for k in on)
            if self.mechset.name == "mainen" and 0 in on:
                P -= 1  # cao_ca is not read by the channel code
            total += 8 * (1 + S) + 8 + 4 * P
        return total


def cable_coefficients(parent: np.ndarray, length_um: np.ndarray, diam_um: np.ndarray,
                       ra_ohm_cm: np.ndarray | float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Axial coupling of cylinder compartments, NEURON's discretisation.

    Half-compartment resistance r_i = 1e-2 * Ra * (L_i/2) / (pi d_i^2 / 4)
    [MOhm]; node-to-parent conductance g = 1/(r_i + r_p) [uS]; with areas
    A = pi d L [um2]:  a_i = -100 g / A_i (row i),  b_i = -100 g / A_p (row
    parent) in S/cm2 -- the same 1e2 factor and signs NEURON writes into
    NODEB / NODEA and the reference's Fmatrix.csv carries.
    Returns (a, b, area)."""
    n = parent.shape[0]
    ra = np.broadcast_to(np.asarray(ra_ohm_cm, dtype=np.float64), (n,))
    area = np.pi * diam_um * length_um
    rhalf = 1e-2 * ra * (length_um / 2.0) / (np.pi * diam_um ** 2 / 4.0)
    a = np.zeros(n)
    b = np.zeros(n)
    for i in range(1, n):
        p = parent[i]
        g = 1.0 / (rhalf[i] + rhalf[p])
        a[i] = -100.0 * g / area[i]
        b[i] = -100.0 * g / area[p]
    return a, b, area


@dataclass
class SectionSpec:
    parent: int          # parent section index (-1 for the root section)
    n_comp: int
    length_um: float     # per compartment
    diam_um: float
    region: int


def expand_sections(secs: list[SectionSpec]) -> tuple[np.ndarray, np.ndarray, np.ndarray,
                                                         np.ndarray, np.ndarray]:
    """Lay sections out as nodes in depth-first preorder.

    Preorder keeps each section's compartments consecutive and makes the
    first child of every node node+1, which maximises the chains the
    simulation kernel passes through registers.  A child section attaches to
    the last compartment (the 1-end) of its parent section.
    Returns (parent, section, length, diam, region_of_section)."""
    kids: dict[int, list[int]] = {}
    roots = []
    for s, sp in enumerate(secs):
        if sp.parent < 0:
            roots.append(s)
        else:
            kids.setdefault(sp.parent, []).append(s)
    if len(roots) != 1:
        raise ValueError("exactly one root section required")
    parent, section, length, diam = [], [], [], []
    last_node = {}
    stack = [roots[0]]
    while stack:
        s = stack.pop()
        sp = secs[s]
        attach = -1 if sp.parent < 0 else last_node[sp.parent]
        for k in range(sp.n_comp):
            node = len(parent)
            parent.append(attach if k == 0 else node - 1)
            section.append(s)
            length.append(sp.length_um)
            diam.append(sp.diam_um)
        last_node[s] = len(parent) - 1
        stack.extend(reversed(kids.get(s, [])))
    region = np.array([sp.region for sp in secs], dtype=np.int32)
    return (np.array(parent, dtype=np.int32), np.array(section, dtype=np.int32),
            np.array(length), np.array(diam), region)


def build_model(secs: list[SectionSpec], mechset: MechSet, region_names: tuple[str, ...],
                region_mechs: dict[str, tuple[str, ...]], ra: float = 100.0,
                cm_of_region: dict[str, float] | None = None, meta: dict | None = None) -> CellModel:
    parent, section, length, diam, sec_region = expand_sections(secs)
    a, b, area = cable_coefficients(parent, length, diam, ra)
    n = parent.shape[0]
    cm = np.ones(n)
    mask = np.zeros((mechset.n_mech, n), dtype=np.uint8)
    for i in range(n):
        rname = region_names[sec_region[section[i]]]
        if cm_of_region and rname in cm_of_region:
            cm[i] = cm_of_region[rname]
        for mname in region_mechs[rname]:
            mask[mechset.mech_index(mname), i] = 1
    m = CellModel(parent=parent, a=a, b=b, cm=cm, section=section, n_sections=len(secs),
                  mechset=mechset, mech_mask=mask, area=area, region=sec_region,
                  region_names=region_names, meta=dict(meta or {}))
    m.meta.setdefault("length_um", length)
    m.meta.setdefault("diam_um", diam)
    m.validate()
    return m


def random_subtree(rng: np.random.Generator, parent_sec: int, n_target: int, region: int,
                   comp_len: float, diam0: float, taper: float, nseg_range: tuple[int, int],
                   out: list[SectionSpec], diam_min: float = 0.4) -> int:
    """Grow a random binary-branching subtree of about n_target compartments
    below ``parent_sec``; returns the number of compartments added."""
    added = 0
    frontier = [(parent_sec, diam0)]
    while added < n_target and frontier:
        k = int(rng.integers(0, len(frontier)))
        psec, d = frontier.pop(k)
        nseg = int(rng.integers(nseg_range[0], nseg_range[1] + 1))
        nseg = min(nseg, n_target - added)
        out.append(SectionSpec(psec, nseg, comp_len, max(d, diam_min), region))
        sidx = len(out) - 1
        added += nseg
        dchild = max(d * taper, diam_min)
        frontier.append((sidx, dchild))
        frontier.append((sidx, dchild))
    return added


def random_binary_cable(rng: np.random.Generator, n_comp: int, comp_len: float,
                        diam_range: tuple[float, float]) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Random binary tree of single-compartment nodes (each picks a parent
    with fewer than two children), relabelled in depth-first preorder.
    Returns (parent, length, diam)."""
    par = np.full(n_comp, -1, dtype=np.int64)
    nkids = np.zeros(n_comp, dtype=np.int64)
    for i in range(1, n_comp):
        cand = np.nonzero(nkids[:i] < 2)[0]
        p = int(cand[rng.integers(0, cand.size)])
        par[i] = p
        nkids[p] += 1
    kids: dict[int, list[int]] = {}
    for i in range(1, n_comp):
        kids.setdefault(int(par[i]), []).append(i)
    order, stack = [], [0]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(reversed(kids.get(v, [])))
    newid = np.empty(n_comp, dtype=np.int64)
    newid[np.array(order)] = np.arange(n_comp)
    parent = np.full(n_comp, -1, dtype=np.int32)
    for old in range(1, n_comp):
        parent[newid[old]] = newid[par[old]]
    diam = rng.uniform(diam_range[0], diam_range[1], n_comp)
    length = np.full(n_comp, comp_len)
    return parent, length, diam


def to_ffi_model(m: CellModel):
    """Create the libngpu model handle (caller destroys it)."""
    import ctypes as C
    m.validate()
    L = _ffi.lib()
    h = C.c_void_p()
    parent = np.ascontiguousarray(m.parent, dtype=np.int32)
    a = np.ascontiguousarray(m.a, dtype=np.float64)
    b = np.ascontiguousarray(m.b, dtype=np.float64)
    cm = np.ascontiguousarray(m.cm, dtype=np.float64)
    sec = np.ascontiguousarray(m.section, dtype=np.int32)
    mask = np.ascontiguousarray(m.mech_mask, dtype=np.uint8)
    _ffi.check("ngpu_model_create", L.ngpu_model_create(
        m.n_nodes, _ffi.ptr(parent), _ffi.ptr(a), _ffi.ptr(b), _ffi.ptr(cm), _ffi.ptr(sec),
        m.n_sections, m.mechset.id, _ffi.ptr(mask), C.byref(h)))
    return h


__all__ = ["CellModel", "SectionSpec", "build_model", "cable_coefficients", "expand_sections",
           "random_subtree", "random_binary_cable", "to_ffi_model", "BY_ID"]
