"""The reference's file formats at the simulation boundary.

A reference run reads its whole problem from the Data/ directory
(GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/Util.h:44-56) and writes one trace
file; these readers / writers keep that contract so existing directories run
unchanged:

* BasicConstSegP.csv -- topology and per-node constants, one comma-terminated
  line per field, written by NeuroGPU_Base/scripts/pyscripts/
  create_auxilliary_data_3.py:229-271 and read by src/MainC.cu:335-551.
* AllParams.csv (src/Util.cu:210-234): line 1 = NSets, then one row of
  NCOMPS*NPARAMS values per set, parameter-major (param_macro,
  src/CudaStuff.cu:212).  ParamsM.csv, the per-model default written by the
  porting step, holds one set section-major (NPARAMS values per section).
* Sim.csv (src/Util.cu:394-432): v_init, dt, NRecSites, RecSites.
* Stim_meta.csv (src/Util.cu:337-358): NStimuli, Nt, comp, loc (1-based), area.
* Stim_raw.csv / Stim_raw<dev>.csv: one row of Nt amplitudes (nA) per stimulus.
* times.csv: Nt per-step dt (ms) -- the step dt the reference uses
  (src/CudaStuff.cu:228-230).
* VHotP<dev>.dat (src/Util.cu:458-476): int32 N, int32 3, N float64 values in
  [set][stim][site][t] order.  RunTimes.csv: "NSets,ms".
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .mechsets import MAINEN, TTPC, MechSet
from .model import CellModel

# BasicConstSegP.csv line numbers (1-based), create_auxilliary_data_3.py:229-264
BCS_FIELDS = ("N", "NComps", "e", "f", "Ks", "SegToComp", "Cms", "NModels", "boolModel",
              "SonNoVec", "Depth", "LognDepth", "nFathers", "nCallForFather", "RelStarts",
              "RelEnds", "RelVec", "SegStartI", "SegEndI", "Fathers", "FIdxs", "CompDepth",
              "CompFDepth", "CompByLevel32", "CompByFLevel32", "nLRel", "LRelStarts",
              "LRelEnds", "nFLRel", "FLRelStarts", "FLRelEnds", "KsB")


def _csv_line(line: str) -> np.ndarray:
    vals = [v for v in line.strip().split(",") if v.strip()]
    return np.array([float(v) for v in vals], dtype=np.float64)


def ref_atof(tok: str) -> np.float32:
    """One AllParams.csv value parsed the way the reference parses it
    (src/Util.cu:143-185, myatof): mantissa digits accumulated in float32
    (each step computed in double and rounded), divided in float32 by the
    float32 power of ten of the fraction digits, then divided or multiplied by
    the C int 10**exp (32-bit, wrapping).  It can land one ulp away from a
    correctly rounded parse, so a drop-in reader must reproduce it to see the
    reference's parameters bit for bit.  A nonzero exponent without a sign is
    rejected: the reference reads an uninitialised sign there."""
    s = tok.lstrip()
    n = len(s)
    i = 0
    sign = np.float32(-1.0 if s[:1] == "-" else 1.0)
    if s[:1] in ("+", "-") and n:
        i = 1
    val, pw = np.float32(0.0), np.float32(1.0)
    while i < n and s[i].isdigit():
        val = np.float32(10.0 * float(val) + (ord(s[i]) - 48))
        i += 1
    if i < n and s[i] == ".":
        i += 1
    while i < n and s[i].isdigit():
        val = np.float32(10.0 * float(val) + (ord(s[i]) - 48))
        pw = np.float32(10.0 * float(pw))
        i += 1
    if i < n and s[i] in "eE":
        i += 1
    esign = None
    if i < n and s[i] in "+-":
        esign = s[i]
        i += 1
    exp = 0
    while i < n and s[i].isdigit():
        exp = 10 * exp + (ord(s[i]) - 48)
        i += 1
    if esign is None and exp != 0:
        raise ValueError(f"value {tok!r}: exponent without a sign")
    p10 = 1
    for _ in range(exp):
        p10 = (p10 * 10 + 2 ** 31) % 2 ** 32 - 2 ** 31
    q = sign * np.float32(val / pw)
    return np.float32(q / np.float32(p10)) if esign == "-" else np.float32(q * np.float32(p10))


def _ref_atof_line(line: str) -> np.ndarray:
    toks = [t for t in line.split(",") if t.strip()]
    uniq, inv = np.unique(np.array(toks), return_inverse=True)
    return np.array([ref_atof(t) for t in uniq], dtype=np.float32)[inv]


def read_basic_const_segp(path: str | os.PathLike) -> dict[str, np.ndarray]:
    """All 32 fields of a BasicConstSegP.csv as float64 arrays."""
    lines = Path(path).read_text().splitlines()
    if len(lines) < len(BCS_FIELDS):
        raise ValueError(f"{path}: expected {len(BCS_FIELDS)} lines, found {len(lines)}")
    return {name: _csv_line(lines[k]) for k, name in enumerate(BCS_FIELDS)}


def parent_from_ks(ks: np.ndarray) -> np.ndarray:
    """Node-order parent vector from the reversed 1-based Ks field: the parent
    of node i > 0 is N - Ks[N - i] (the kernel's parentIndex,
    src/CudaStuff.cu:195); the root's is -1."""
    n = ks.size
    parent = np.full(n, -1, dtype=np.int32)
    for i in range(1, n):
        parent[i] = n - int(ks[n - i])
    return parent


def son_no_vec(parent: np.ndarray) -> np.ndarray:
    """Child rank of every node under its parent, in node order, with the
    root's set to 0 (create_auxilliary_data_3.py:72-84)."""
    used = np.zeros(parent.size, dtype=np.int64)
    out = np.zeros(parent.size, dtype=np.int64)
    for i in range(parent.size):
        p = 0 if i == 0 else parent[i]
        used[p] += 1
        out[i] = used[p]
    out[0] = 0
    return out


def ancestor_table(ks: np.ndarray) -> np.ndarray:
    """The pointer-jumping table FIdxs of the reference's back-substitution
    (create_auxilliary_data_3.py:53-67): row k holds, for every reversed
    1-based node index, the 1-based index of its 2^k-th ancestor (N+1 past the
    root); rows stop before the table saturates."""
    n = ks.size
    father = np.concatenate([ks[1:], [n + 1, n + 1]]).astype(np.int64)
    rows = []
    for lev in range(1, int(np.ceil(np.log2(n))) + 3 + 1):
        cur = np.arange(1, father.size + 1)
        for _ in range(2 ** (lev - 1)):
            cur = father[cur - 1]
        rows.append(cur)
    tab = np.array(rows)
    ind = int(np.nonzero(np.all(tab == tab[-1], axis=1))[0][0]) + 1
    if ind != 0:
        tab = tab[:ind - 1, :]
    return tab[:, :n]


def _starts_ends(groups: list) -> tuple[np.ndarray, np.ndarray]:
    """0-based start / end position of each group in their concatenation."""
    lens = np.array([len(g) for g in groups], dtype=np.int64)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]]) if lens.size else lens
    return starts, starts + lens - 1


def level_schedule(ks: np.ndarray) -> dict:
    """The reference's level schedule of its branched solve over the reversed
    1-based parent field Ks (P/make_tree_from_parent_vec.py:17-59): the
    junction fathers and, per father, the positions that call it; the chain
    segments between calls (SegStartI / SegEndI, 1-based); each segment's
    elimination level and each father's level.  Index arithmetic as there,
    including where it mixes 1-based values and 0-based positions."""
    ks = np.asarray(ks, dtype=np.int64)
    n = ks.size
    pos = np.arange(1, n + 1)
    fathers = np.unique(ks[(ks != pos) & (ks > 0)])
    related = [np.nonzero(ks == fa)[0] for fa in fathers]
    call = np.nonzero(np.isin(ks, fathers))[0] + 1
    r_fathers = np.zeros(int(fathers.max()) if fathers.size else 0)
    r_fathers[fathers - 1] = np.arange(1, fathers.size + 1)
    seg_start = np.concatenate([[2], call + 1])
    seg_end = np.concatenate([call - 1, [n - 1]])
    level = np.zeros(seg_start.size, dtype=np.int64)
    level[np.isin(seg_start - 1, fathers)] = 1
    for lv in range(1, 51):
        calls_to = ks[seg_end[level == lv]]
        level[np.isin(seg_start - 1, calls_to)] = lv + 1
    flevel = np.ones(fathers.size, dtype=np.int64)
    for lv in range(1, int(level.max()) + 1):
        calls_to = ks[seg_end[level == lv]]
        # a (1, m) index array of positions minus one, as the reference forms it
        sel = np.subtract(np.where(calls_to <= fathers.max()), 1)
        which = r_fathers[np.subtract(calls_to[sel], 1)][0]
        flevel[which.astype(np.int64) - 1] = lv + 1
    seg_end[-1] = n
    rel_starts, rel_ends = _starts_ends(related)
    return {"fathers": fathers, "related": related, "rel_starts": rel_starts, "rel_ends": rel_ends,
            "rel_vec": np.concatenate(related) if related else np.zeros(0, np.int64), "call": call,
            "seg_start": seg_start, "seg_end": seg_end, "level": level, "flevel": flevel,
            "depth": int(level.max())}


def _by_level32(levels: np.ndarray, targets) -> tuple[np.ndarray, list]:
    """Rows of 32 (1-based) indices per level, the last index repeated to fill
    a row; the 1-based row numbers of each level."""
    rows, related = [], []
    for lv in targets:
        comps = np.nonzero(levels == lv)[0] + 1
        k = int(np.ceil(comps.size / 32.0))
        padded = np.full(k * 32, comps[-1])
        padded[:comps.size] = comps
        first = len(rows) + 1
        rows += list(padded.reshape(k, 32))
        related.append(list(range(first, len(rows) + 1)))
    return (np.array(rows) if rows else np.zeros((0, 32))), related


def basic_const_fields(ks: np.ndarray, e: np.ndarray, f: np.ndarray, seg_to_comp: np.ndarray, cms: np.ndarray,
                       bool_model: np.ndarray, n_comps: int) -> dict[str, np.ndarray]:
    """All 32 fields of BasicConstSegP.csv from the model's reversed parent
    field Ks, coefficients e / f (reversed B / A columns of NEURON's matrix),
    node-to-compartment map, capacitances and mechanism flags [n_models][N]:
    the auxiliary data the reference's solver reads
    (P/create_auxilliary_data_3.py:22-271, with
    P/make_tree_from_parent_vec.py); uint16 fields wrap as there."""
    ks = np.asarray(ks, dtype=np.int64)
    n = ks.size
    parent = parent_from_ks(ks)
    sons = son_no_vec(parent)
    if sons.max() > 2:  # the reference's solver allows two children per node (create_auxilliary_data_3.py:83)
        raise ValueError("a node has more than two children: the reference's format cannot hold the tree")
    fidx = ancestor_table(ks)
    sch = level_schedule(ks)
    depth = sch["depth"]
    level, flevel = sch["level"], sch["flevel"]
    last_level_i = int(np.nonzero(level == level.max())[0][0]) + 1
    ksb = np.concatenate([ks, [sch["seg_end"][last_level_i - 1]]])
    comp32, lrel = _by_level32(level, range(depth + 1))
    fcomp32, flrel = _by_level32(flevel, range(1, depth + 1)) if depth > 0 else (np.zeros((0, 32)), [])
    ls, le = _starts_ends(lrel)
    fs, fe = _starts_ends(flrel) if depth > 0 else (np.zeros(0), np.zeros(0))
    u16 = lambda x: np.asarray(x, dtype=np.int64).astype(np.uint16).astype(np.float64)
    bm = np.asarray(bool_model, dtype=np.float64)
    return {
        "N": np.array([n], dtype=np.float64), "NComps": np.array([n_comps], dtype=np.float64),
        "e": np.asarray(e, dtype=np.float64), "f": np.asarray(f, dtype=np.float64), "Ks": u16(ks),
        "SegToComp": u16(seg_to_comp), "Cms": np.asarray(cms, dtype=np.float64),
        "NModels": np.array([bm.shape[0]], dtype=np.float64), "boolModel": bm.reshape(-1),
        "SonNoVec": u16(sons), "Depth": np.array([depth], dtype=np.float64),
        "LognDepth": np.array([fidx.shape[0]], dtype=np.float64),
        "nFathers": np.array([sch["fathers"].size], dtype=np.float64),
        "nCallForFather": np.array([sch["call"].size], dtype=np.float64),
        "RelStarts": u16(sch["rel_starts"] + 1), "RelEnds": u16(sch["rel_ends"] + 1),
        "RelVec": u16(sch["rel_vec"] + 1), "SegStartI": u16(sch["seg_start"]), "SegEndI": u16(sch["seg_end"]),
        "Fathers": u16(sch["fathers"]), "FIdxs": u16(fidx.reshape(-1)),
        "CompDepth": np.array([comp32.shape[0]], dtype=np.float64),
        "CompFDepth": np.array([fcomp32.shape[0]], dtype=np.float64),
        "CompByLevel32": u16(comp32.reshape(-1)), "CompByFLevel32": u16(fcomp32.reshape(-1)),
        "nLRel": np.array([len(lrel)], dtype=np.float64), "LRelStarts": u16(ls), "LRelEnds": u16(le),
        "nFLRel": np.array([len(flrel)], dtype=np.float64), "FLRelStarts": u16(fs), "FLRelEnds": u16(fe),
        "KsB": u16(ksb - 1),
    }


def format_basic_const_segp(fields: dict[str, np.ndarray]) -> str:
    """The file text: one line per field, every value as %.9f followed by a
    comma (P/create_auxilliary_data_3.py:262-271)."""
    return "".join("".join(f"{x:.9f}," for x in np.asarray(fields[k]).reshape(-1)) + "\n" for k in BCS_FIELDS)


def ks_from_parent(parent: np.ndarray) -> np.ndarray:
    """Inverse of parent_from_ks: the reversed 1-based parent field."""
    n = parent.size
    ks = np.zeros(n, dtype=np.int64)
    for j in range(1, n):
        ks[j] = n - int(parent[n - j])
    return ks


def write_basic_const_segp(path: str | os.PathLike, cell: CellModel, bool_model: np.ndarray | None = None) -> None:
    """BasicConstSegP.csv of a CellModel (node order: Hines, root 0), for the
    reference's simulator or this library's command line.  bool_model: the
    file's mechanism rows [n_models][N] (default: the cell's mechanism mask)."""
    n = cell.n_nodes
    ks = ks_from_parent(np.asarray(cell.parent))
    f = np.asarray(cell.a, dtype=np.float64)[::-1].copy()
    e = np.asarray(cell.b, dtype=np.float64)[::-1].copy()
    bm = np.asarray(cell.mech_mask if bool_model is None else bool_model, dtype=np.float64)
    fields = basic_const_fields(ks, e, f, np.asarray(cell.section), np.asarray(cell.cm), bm, cell.n_sections)
    Path(path).write_text(format_basic_const_segp(fields))


@dataclass
class ReferenceModel:
    """A reference Data/ directory turned into the library's inputs."""
    cell: CellModel
    params: np.ndarray          # [n_sets, n_params, n_sections] float32 (library mechanism set)
    amps: np.ndarray            # [n_stim, nt] float32
    dts: np.ndarray             # [nt] float32
    stim_node: int              # 0-based node
    stim_area: float            # um2 (float32 value)
    rec_nodes: np.ndarray       # int32
    v_init: float
    raw: dict = field(default_factory=dict)


def mechset_for(n_models: int, n_params: int, mechset=None) -> tuple[MechSet, list[int], list[int] | None]:
    """Library mechanism set for a reference build, the library mechanism of
    each of the file's boolModel rows, and (when the reference build's
    parameter list differs) the library parameter index of each file
    parameter.  A set given as `mechset` (e.g. one generated from the
    model's .mod files, whose mechanism and parameter order is the reference
    build's) is taken as is when its sizes match the files'."""
    if mechset is not None:
        if mechset.n_mech != n_models or mechset.n_params != n_params:
            raise ValueError(f"mechanism set {getattr(mechset, 'name', '?')} has {mechset.n_mech} mechanisms and "
                             f"{mechset.n_params} parameters; the files have {n_models} and {n_params}")
        return mechset, list(range(n_models)), None
    if n_params == TTPC.n_params and n_models == TTPC.n_mech:
        return TTPC, list(range(TTPC.n_mech)), None
    if n_params == MAINEN.n_params and n_models <= MAINEN.n_mech:
        # the Mainen build writes 7 boolModel rows: ca cad kca km kv na pas
        return MAINEN, list(range(n_models)), None
    if n_params == 2 and n_models == 1:
        # single-mechanism passive build (Figures/FigureS3_passive/CParsed): pas
        return TTPC, [TTPC.mech_index("pas")], [TTPC.param_index("g_pas"), TTPC.param_index("e_pas")]
    raise ValueError(f"no library mechanism set matches a build with {n_models} mechanisms "
                     f"and {n_params} parameters")


def cell_from_basic_const(bc: dict[str, np.ndarray], n_params: int, mechset=None) -> CellModel:
    n = int(bc["N"][0])
    ncomps = int(bc["NComps"][0])
    nmod = int(bc["NModels"][0])
    ms, mech_map, _ = mechset_for(nmod, n_params, mechset)
    parent = parent_from_ks(bc["Ks"])
    e, f = bc["e"], bc["f"]
    a = f[::-1][:n].copy()        # the reference's f, reversed into node order
    b = e[::-1][:n].copy()
    a[0] = 0.0
    b[0] = 0.0
    bool_model = bc["boolModel"].reshape(nmod, n)
    mask = np.zeros((ms.n_mech, n), dtype=np.uint8)
    for row, k in enumerate(mech_map):
        mask[k] = (bool_model[row] != 0)
    cell = CellModel(parent=parent, a=a, b=b, cm=bc["Cms"].astype(np.float64).copy(),
                     section=bc["SegToComp"].astype(np.int32), n_sections=ncomps,
                     mechset=ms, mech_mask=mask)
    cell.validate()
    return cell


def read_params_csv(path: str | os.PathLike, n_comps: int, n_params: int, has_count: bool) -> np.ndarray:
    """AllParams.csv (has_count: first line = NSets, rows parameter-major,
    values parsed like the reference's myatof) or ParamsM.csv (one
    section-major row) -> [n_sets, n_params, n_comps] float32 in the file's
    own parameter order."""
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    if has_count:
        n_sets = int(float(lines[0].split(",")[0]))
        rows = lines[1:1 + n_sets]
    else:
        rows = lines
    out = np.zeros((len(rows), n_params, n_comps), dtype=np.float32)
    for k, ln in enumerate(rows):
        v = (_ref_atof_line(ln) if has_count else _csv_line(ln))[:n_params * n_comps]
        if v.size != n_params * n_comps:
            raise ValueError(f"{path}: row {k} has {v.size} values, expected {n_params * n_comps}")
        out[k] = v.reshape(n_params, n_comps) if has_count else v.reshape(n_comps, n_params).T
    return out


def write_allparams_csv(path: str | os.PathLike, params: np.ndarray) -> None:
    """AllParams.csv in the reference's format (NeuroGPU_Base/scripts/
    template/extractModel_mappings.py:326-330): the set count, then one
    '%.5E, '-separated row per set."""
    with open(path, "w") as fh:
        fh.write(f"{params.shape[0]},\n")
        for p in params.reshape(params.shape[0], -1):
            fh.write(", ".join(f"{x:.5E}" for x in p) + ",\n")


def map_params(file_params: np.ndarray, n_models: int, ms_params: int, mechset=None) -> np.ndarray:
    """File parameter order -> library mechanism-set order."""
    ms, _, pmap = mechset_for(n_models, file_params.shape[1], mechset)
    if pmap is None:
        return file_params
    out = np.zeros((file_params.shape[0], ms.n_params, file_params.shape[2]), dtype=np.float32)
    for j, k in enumerate(pmap):
        out[:, k, :] = file_params[:, j, :]
    return out


def read_sim_csv(path: str | os.PathLike) -> tuple[float, float, np.ndarray]:
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    v_init = float(_csv_line(lines[0])[0])
    dt = float(_csv_line(lines[1])[0])
    n_rec = int(_csv_line(lines[2])[0])
    rec = _csv_line(lines[3])[:n_rec].astype(np.int32) if n_rec else np.zeros(0, np.int32)
    return v_init, dt, rec


def read_stim_meta(path: str | os.PathLike) -> tuple[int, int, int, float]:
    """(n_stim, nt, loc as a 0-based node, area)."""
    v = [float(ln.split(",")[0]) for ln in Path(path).read_text().splitlines() if ln.strip()]
    return int(v[0]), int(v[1]), int(v[3]) - 1, float(np.float32(v[4]))


def read_rows(path: str | os.PathLike, n_rows: int, n_cols: int) -> np.ndarray:
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    out = np.zeros((n_rows, n_cols), dtype=np.float32)
    for k in range(n_rows):
        v = _csv_line(lines[k])[:n_cols]
        out[k, :v.size] = v
    return out


def read_data_dir(data: str | os.PathLike, stim_index: int | None = None,
                  params_file: str | None = None, mechset=None) -> ReferenceModel:
    """Everything a reference run reads from its Data/ directory.  stim_index:
    the device / stimulus number the reference appends to Stim_raw (argv[1],
    src/Util.cu:359-364); None reads Stim_raw.csv.  mechset: the model's
    mechanism set when it is none of the built-in ones (a set generated from
    the model's .mod files by nmodl.generate_from_files, registered)."""
    d = Path(data)
    bc = read_basic_const_segp(d / "BasicConstSegP.csv")
    n_comps = int(bc["NComps"][0])
    n_models = int(bc["NModels"][0])
    n_nodes = int(bc["N"][0])
    if params_file is None:
        params_file = "AllParams.csv" if (d / "AllParams.csv").exists() and \
            not (d / "AllParams.csv").read_text().startswith("version https://git-lfs") else "ParamsM.csv"
    has_count = Path(params_file).name.startswith("AllParams")
    # parameter count of the build: the row length over NComps
    first = [ln for ln in (d / params_file).read_text().splitlines() if ln.strip()]
    row = first[1] if has_count else first[0]
    n_params = _csv_line(row).size // n_comps
    fparams = read_params_csv(d / params_file, n_comps, n_params, has_count)
    cell = cell_from_basic_const(bc, n_params, mechset)
    params = map_params(fparams, n_models, n_params, mechset)
    v_init, _, rec = read_sim_csv(d / "Sim.csv")
    n_stim, nt, loc, area = read_stim_meta(d / "Stim_meta.csv")
    raw_name = "Stim_raw.csv" if stim_index is None else f"Stim_raw{stim_index}.csv"
    amps = read_rows(d / raw_name, n_stim, nt)
    dts = read_rows(d / "times.csv", 1, nt)[0]
    if not (0 <= loc < n_nodes):
        raise ValueError(f"stimulus location {loc + 1} outside the {n_nodes}-node tree")
    return ReferenceModel(cell, params, amps, dts, loc, area, rec, v_init,
                          raw={"basic_const": bc, "file_params": fparams})


def write_data_dir(data: str | os.PathLike, cell: CellModel, params: np.ndarray, amps: np.ndarray,
                   dts: np.ndarray, stim_node: int, stim_area: float, rec_nodes, v_init: float, dt: float,
                   bool_model: np.ndarray | None = None, stim_index: int | None = None,
                   param_index=None) -> None:
    """A reference Data/ directory for a model: BasicConstSegP.csv,
    AllParams.csv, Sim.csv, Stim_meta.csv, Stim_raw[<stim_index>].csv and
    times.csv, in the formats read_data_dir (and the reference's reader,
    src/MainC.cu:335-551, src/Util.cu) reads.  params [n_sets, n_params,
    n_sections] in the library mechanism set's order; param_index: the
    library parameter index of each parameter the reference build lists
    (default: all, in order; the inverse of map_params); amps [n_stim, nt]
    nA; dts [nt] ms.  AllParams.csv holds 6 significant digits, as the
    reference's writer prints them."""
    d = Path(data)
    d.mkdir(parents=True, exist_ok=True)
    write_basic_const_segp(d / "BasicConstSegP.csv", cell, bool_model)
    params = np.asarray(params, dtype=np.float32)
    if param_index is not None:
        params = params[:, np.asarray(param_index, dtype=np.int64), :]
    write_allparams_csv(d / "AllParams.csv", params)
    rec = [int(r) for r in np.asarray(rec_nodes).reshape(-1)]
    (d / "Sim.csv").write_text(f"{v_init:.5f},\n{dt:.5f},\n{len(rec):.5f},\n" +
                              "".join(f"{r:.5f}," for r in rec) + "\n")
    amps = np.asarray(amps, dtype=np.float32)
    (d / "Stim_meta.csv").write_text(f"{amps.shape[0]}\n{amps.shape[1]}\n0\n{stim_node + 1}\n{stim_area!r}\n")
    raw = "Stim_raw.csv" if stim_index is None else f"Stim_raw{stim_index}.csv"
    (d / raw).write_text("".join("".join(f"{x:.6f}," for x in row) + "\n" for row in amps))
    (d / "times.csv").write_text("".join(f"{x:.5f}," for x in np.asarray(dts, dtype=np.float64)) + "\n")


def write_vhot(path: str | os.PathLike, traces: np.ndarray) -> None:
    """VHotP<dev>.dat: int32 count, int32 3, then float64 values."""
    flat = np.ascontiguousarray(traces, dtype=np.float64).reshape(-1)
    with open(path, "wb") as fh:
        np.array([flat.size, 3], dtype=np.int32).tofile(fh)
        flat.tofile(fh)


def read_vhot(path: str | os.PathLike) -> np.ndarray:
    """nrnMread of Figures/Figure4_DEAP/neurogpu_multistim_evaluator_par.py:
    42-46 (the type word is ignored, values are float64)."""
    with open(path, "rb") as fh:
        n, _typ = np.fromfile(fh, dtype=np.int32, count=2)
        return np.fromfile(fh, dtype=np.float64, count=int(n))


def write_run_times(path: str | os.PathLike, n_sets: int, ms: float) -> None:
    Path(path).write_text(f"{n_sets},{ms:f}\n")
