"""ctypes binding of the CPU oracle (liboracle.so) and of the reference's own
channel functions built by build_ref.sh (oracle/_ref/libref_*.so).

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
the CPU-baseline / reference arm of bench.py; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
# the reference project's source tree, read by the pins and fixture scripts
# where it is present (the same variable and default as build_ref.sh)
REFERENCE_DIR = Path(os.environ.get("NGPU_REFERENCE_DIR", "/root/reference"))

MECHSET_TTPC = 0
MECHSET_MAINEN = 1
FLAG_FD = 1


class _Model(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("parent", C.c_void_p), ("a", C.c_void_p),
                ("b", C.c_void_p), ("cm", C.c_void_p), ("section", C.c_void_p),
                ("n_sections", C.c_int), ("mechset", C.c_int), ("mech_mask", C.c_void_p)]


_lib = None


def build() -> Path:
    """make liboracle.so (no-op when up to date)."""
    src = [HERE / "oracle.c", HERE / "oracle.h"]
    if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        P, I, D = C.c_void_p, C.c_int, C.c_double
        for nm in ("ong_run_f64", "ong_run_f32"):
            f = getattr(L, nm)
            f.restype = I
            f.argtypes = [P, I, P, I, I, P, P, I, D, I, P, D, I, P, I]
        for nm in ("ong_n_params", "ong_n_states", "ong_n_mechs"):
            getattr(L, nm).restype = I
            getattr(L, nm).argtypes = [I]
        L.ong_node_init_f64.argtypes = [I, P, D, P, P]
        L.ong_node_deriv_f64.argtypes = [I, P, D, D, P, P]
        L.ong_node_current_f64.argtypes = [I, P, D, P, P, P]
        L.ong_node_current_f64.restype = D
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def run(parent, a, b, cm, section, n_sections, mechset, mech_mask, params, amps, dts, stim_node,
        stim_area, rec_nodes, v_init, precision: str = "f64", fd: bool = True,
        n_threads: int = 0) -> np.ndarray:
    """Oracle simulation; returns V [n_sets, n_stim, n_rec, nt] (float64)."""
    keep = dict(parent=np.ascontiguousarray(parent, dtype=np.int32),
                a=np.ascontiguousarray(a, dtype=np.float64),
                b=np.ascontiguousarray(b, dtype=np.float64),
                cm=np.ascontiguousarray(cm, dtype=np.float64),
                section=np.ascontiguousarray(section, dtype=np.int32),
                mask=np.ascontiguousarray(mech_mask, dtype=np.uint8))
    m = _Model(int(keep["parent"].size), _p(keep["parent"]), _p(keep["a"]), _p(keep["b"]),
               _p(keep["cm"]), _p(keep["section"]), int(n_sections), int(mechset), _p(keep["mask"]))
    pr = np.ascontiguousarray(params, dtype=np.float32)
    am = np.ascontiguousarray(np.atleast_2d(amps), dtype=np.float32)
    nt = am.shape[1]
    dd = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float32), (nt,)))
    rec = np.ascontiguousarray(np.asarray(rec_nodes, dtype=np.int32).reshape(-1))
    out = np.zeros((pr.shape[0], am.shape[0], rec.size, nt), dtype=np.float64)
    fn = lib().ong_run_f64 if precision == "f64" else lib().ong_run_f32
    rc = fn(C.byref(m), pr.shape[0], _p(pr), am.shape[0], nt, _p(am), _p(dd), int(stim_node),
            float(stim_area), rec.size, _p(rec), float(v_init), FLAG_FD if fd else 0, _p(out),
            int(n_threads))
    if rc != 0:
        raise ValueError(f"oracle rejected the input ({rc})")
    return out


def run_workload(w, precision: str = "f64", fd: bool = True, n_threads: int = 0) -> np.ndarray:
    """Oracle run of a neurogpu_b200.configs.Workload-like object."""
    c = w.cell
    return run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask,
               w.params, w.amps, w.dts, w.stim_node, w.stim_area, w.rec_nodes, w.v_init,
               precision=precision, fd=fd, n_threads=n_threads)


# ---- the reference's own channel functions (oracle/_ref, built by build_ref.sh) ----
def ref_channels(mechset: int) -> C.CDLL | None:
    name = "libref_ttpc.so" if mechset == MECHSET_TTPC else "libref_mainen.so"
    path = REF_DIR / name
    if not path.exists():
        return None
    L = C.CDLL(str(path))
    fn = L.ref_ttpc_mech if mechset == MECHSET_TTPC else L.ref_mainen_mech
    fn.restype = C.c_double
    fn.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def ref_binary() -> Path | None:
    p = REF_DIR / "neuroGPU_ttpc512"
    return p if p.exists() and os.access(p, os.X_OK) else None
