"""Python front end of the simulation core (a thin layer over include/ngpu.h).

``run`` is the drop-in for one reference ``neuroGPU`` process
(GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/kernel.cu:8-33 -> RunByModelP ->
stEfork2Main, src/CudaStuff.cu:518-587): parameters, stimuli and recording
sites in, voltage traces out, with the reference's array layouts.
``Simulator`` keeps the simulation resident on the GPU between calls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .model import CellModel, to_ffi_model

_PREC = {"fp32": _ffi.NGPU_FP32, "fp64": _ffi.NGPU_FP64}


def _stream_ptr(stream) -> C.c_void_p | None:
    if stream is None:
        return None
    h = getattr(stream, "cuda_stream", stream)
    return C.c_void_p(int(h))


def _as_f32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


class Model:
    """libngpu model handle for a :class:`CellModel`."""

    def __init__(self, cell: CellModel):
        self.cell = cell
        self._h = to_ffi_model(cell)

    @property
    def handle(self):
        return self._h

    def layout(self) -> dict:
        L = _ffi.lib()
        sr, pr, nj = C.c_int32(), C.c_int32(), C.c_int32()
        sv, prd = C.c_int64(), C.c_int64()
        _ffi.check("ngpu_model_layout", L.ngpu_model_layout(self._h, C.byref(sr), C.byref(pr),
                                                            C.byref(nj), C.byref(sv), C.byref(prd)))
        return {"state_rows": sr.value, "param_rows": pr.value, "n_jslots": nj.value,
                "state_vars": sv.value, "param_reads": prd.value}

    def partition(self, n_warps: int) -> dict:
        """The tree split a CTA of n_warps warps uses, per node in this model's
        numbering (see ngpu_model_partition)."""
        n = self.cell.n_nodes
        sep, item, js, ps = (np.zeros(n, dtype=np.int32) for _ in range(4))
        nj = C.c_int32()
        _ffi.check("ngpu_model_partition", _ffi.lib().ngpu_model_partition(
            self._h, int(n_warps), _ffi.ptr(sep), _ffi.ptr(item), _ffi.ptr(js), _ffi.ptr(ps), C.byref(nj)))
        return {"sep": sep.astype(bool), "item": item, "jslot": js, "pslot": ps, "n_jslots": nj.value}

    def nodes(self) -> dict:
        """Stiff-edge merging (ngpu_model_nodes): internal node count, the
        internal node of every node of this model, and each node's area over
        its internal node's area."""
        n = self.cell.n_nodes
        ni = C.c_int32()
        node_internal = np.zeros(n, dtype=np.int32)
        scale = np.zeros(n, dtype=np.float64)
        _ffi.check("ngpu_model_nodes", _ffi.lib().ngpu_model_nodes(
            self._h, C.byref(ni), None, _ffi.ptr(node_internal), _ffi.ptr(scale)))
        return {"n_internal": ni.value, "node_internal": node_internal, "density_scale": scale}

    def arrays(self) -> dict:
        """The merged model in internal order (ngpu_model_arrays)."""
        n = self.nodes()["n_internal"]
        par = np.zeros(n, dtype=np.int32)
        a, b, cm = (np.zeros(n, dtype=np.float64) for _ in range(3))
        _ffi.check("ngpu_model_arrays", _ffi.lib().ngpu_model_arrays(
            self._h, _ffi.ptr(par), _ffi.ptr(a), _ffi.ptr(b), _ffi.ptr(cm)))
        return {"parent": par, "a": a, "b": b, "cm": cm}

    def split_info(self, n_warps: int) -> dict:
        """The split in the library's internal node order (ngpu_model_split_info)."""
        n = self.nodes()["n_internal"]
        L = _ffi.lib()
        nc, ns = C.c_int32(), C.c_int32()
        _ffi.check("ngpu_model_split_info", L.ngpu_model_split_info(
            self._h, int(n_warps), None, C.byref(nc), None, 0, C.byref(ns), None, 0, None, None))
        perm = np.zeros(n, dtype=np.int32)
        comps = np.zeros((max(1, nc.value), 6), dtype=np.int32)
        seps = np.zeros((max(1, ns.value), 3), dtype=np.int32)
        js, ps = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        _ffi.check("ngpu_model_split_info", L.ngpu_model_split_info(
            self._h, int(n_warps), _ffi.ptr(perm), C.byref(nc), _ffi.ptr(comps), nc.value, C.byref(ns),
            _ffi.ptr(seps), ns.value, _ffi.ptr(js), _ffi.ptr(ps)))
        return {"perm": perm, "comps": comps[:nc.value], "seps": seps[:ns.value], "jslot": js, "pslot": ps}

    def close(self) -> None:
        if self._h:
            _ffi.lib().ngpu_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


LAYOUTS = {"lane": _ffi.NGPU_LAYOUT_LANE_INSTANCE, "warp": _ffi.NGPU_LAYOUT_WARP_INSTANCE}


class Simulator:
    """Resident simulation of n_sets x n_stim instances of one model."""

    def __init__(self, model: Model | CellModel, n_sets: int, n_stim: int, precision: str = "fp32",
                 n_warps: int = 0, items_per_warp: int = 0, layout: str = "lane"):
        """layout "lane" (one lane per instance, 32 instances per CTA; the
        default): n_warps warps per CTA share the tree (1..16; above 8 the
        runtime-compiled kernel, bounded for 3 CTAs per SM), items_per_warp
        work items per warp (1..8).  layout "warp" (one warp per instance, for
        batches too small to fill the GPU): n_warps instances per CTA (1..8),
        items_per_warp the work items the instance's tree is split into
        (1..512).  0 = the library's choice; see neurogpu_b200.autotune for
        timing-based selection."""
        self.model = model if isinstance(model, Model) else Model(model)
        self.n_sets, self.n_stim = int(n_sets), int(n_stim)
        self.precision = precision
        if layout not in LAYOUTS:
            raise ValueError(f"layout must be one of {sorted(LAYOUTS)}")
        h = C.c_void_p()
        _ffi.check("ngpu_sim_create_layout", _ffi.lib().ngpu_sim_create_layout(
            self.model.handle, self.n_sets, self.n_stim, _PREC[precision], LAYOUTS[layout], int(n_warps),
            int(items_per_warp), C.byref(h)))
        self._h = h
        self.nt = 0
        self.n_rec = 1

    def set_params(self, params) -> None:
        """params [n_sets, n_params, n_sections]: numpy (host) or a CUDA tensor."""
        L = _ffi.lib()
        if hasattr(params, "is_cuda") and params.is_cuda:
            t = params.contiguous().float()
            _ffi.check("ngpu_sim_set_params", L.ngpu_sim_set_params(self._h, C.c_void_p(t.data_ptr()), 1))
            self._keep = t
        else:
            p = _as_f32(params)
            cell = self.model.cell
            exp = (self.n_sets, cell.n_params(), cell.n_sections)
            if p.shape != exp:
                raise ValueError(f"params shape {p.shape} != {exp}")
            _ffi.check("ngpu_sim_set_params", L.ngpu_sim_set_params(self._h, _ffi.ptr(p), 0))

    def set_stimulus(self, amps, dts, stim_node: int, stim_area_um2: float) -> None:
        a = _as_f32(amps)
        if a.ndim != 2 or a.shape[0] != self.n_stim:
            raise ValueError("amps must be [n_stim, nt]")
        nt = a.shape[1]
        d = _as_f32(np.broadcast_to(np.asarray(dts, dtype=np.float32), (nt,)))
        _ffi.check("ngpu_sim_set_stimulus", _ffi.lib().ngpu_sim_set_stimulus(
            self._h, nt, _ffi.ptr(a), _ffi.ptr(d), int(stim_node), float(stim_area_um2), 0))
        self.nt = nt

    def set_recording(self, rec_nodes, rec_every: int = 1) -> None:
        r = np.ascontiguousarray(np.asarray(rec_nodes, dtype=np.int32).reshape(-1))
        _ffi.check("ngpu_sim_set_recording", _ffi.lib().ngpu_sim_set_recording(
            self._h, r.size, _ffi.ptr(r), int(rec_every)))
        self.n_rec = int(r.size)

    def init(self, v_init: float, stream=None) -> None:
        _ffi.check("ngpu_sim_init", _ffi.lib().ngpu_sim_init(self._h, float(v_init), _stream_ptr(stream)))

    def advance(self, t0: int, n_steps: int, stream=None) -> None:
        _ffi.check("ngpu_sim_advance", _ffi.lib().ngpu_sim_advance(
            self._h, int(t0), int(n_steps), _stream_ptr(stream)))

    @property
    def n_samples(self) -> int:
        return int(_ffi.lib().ngpu_sim_n_samples(self._h))

    def trace(self, stream=None) -> np.ndarray:
        out = np.empty((self.n_sets, self.n_stim, self.n_rec, self.n_samples), dtype=np.float32)
        _ffi.check("ngpu_sim_get_trace", _ffi.lib().ngpu_sim_get_trace(
            self._h, _ffi.ptr(out), 0, _stream_ptr(stream)))
        return out

    def trace_into(self, dev_ptr: int, stream=None) -> None:
        """Write the trace [n_sets, n_stim, n_rec, n_samples] to device memory."""
        _ffi.check("ngpu_sim_get_trace", _ffi.lib().ngpu_sim_get_trace(
            self._h, C.c_void_p(dev_ptr), 1, _stream_ptr(stream)))

    def features(self, dt: float, stim_on: float, stim_off: float, site: int = 0, threshold: float = -20.0,
                 stream=None):
        """The 20 features of neurogpu_b200.features of every instance's trace
        at recording site `site`, computed where the trace lies
        (ngpu_sim_features): a float32 CUDA tensor [n_sets, n_stim, 20].
        dt: the sample spacing (step dt x rec_every)."""
        import torch
        out = torch.empty((self.n_sets, self.n_stim, 20), dtype=torch.float32, device="cuda")
        _ffi.check("ngpu_sim_features", _ffi.lib().ngpu_sim_features(
            self._h, int(site), float(dt), float(stim_on), float(stim_off), float(threshold),
            C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def dvdt_peaks(self, dt: float, site: int = 0, height: float = 15.0, distance: int = 5, stream=None):
        """Exploration score of every instance's trace at recording site
        `site`, computed where the trace lies (ngpu_sim_dvdt_peaks): the
        number of peaks scipy.signal.find_peaks(diff(v) / dt, height,
        distance) finds; an int32 CUDA tensor [n_sets, n_stim].  dt: the
        sample spacing (step dt x rec_every)."""
        import torch
        L = _ffi.lib()
        need = int(L.ngpu_dvdt_peaks_scratch_bytes(self.n_sets * self.n_stim, self.n_samples))
        scratch = torch.empty(max(need, 4), dtype=torch.uint8, device="cuda")
        out = torch.empty((self.n_sets, self.n_stim), dtype=torch.int32, device="cuda")
        _ffi.check("ngpu_sim_dvdt_peaks", L.ngpu_sim_dvdt_peaks(
            self._h, int(site), float(dt), float(height), int(distance), C.c_void_p(scratch.data_ptr()),
            scratch.numel(), C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        self._keep_scratch = scratch  # until the stream has used it
        return out

    def layout(self) -> dict:
        """{"layout": "lane" | "warp", "cta_warps": .., "items": ..} with the
        library's choices filled in (ngpu_sim_layout)."""
        lay, w, it = C.c_int32(), C.c_int32(), C.c_int32()
        _ffi.check("ngpu_sim_layout", _ffi.lib().ngpu_sim_layout(self._h, C.byref(lay), C.byref(w), C.byref(it)))
        return {"layout": {v: k for k, v in LAYOUTS.items()}[lay.value], "cta_warps": w.value, "items": it.value}

    def param_folds(self) -> int:
        """Parameters compiled into this simulation's kernel as constants
        (after init; see ngpu_sim_param_folds)."""
        n = C.c_int32()
        _ffi.check("ngpu_sim_param_folds", _ffi.lib().ngpu_sim_param_folds(self._h, C.byref(n)))
        return n.value

    def param_rows(self) -> tuple[int, int]:
        """(parameter rows the kernels read, rows the table holds) per group of
        32 instances; see ngpu_sim_param_rows."""
        a, b = C.c_int32(), C.c_int32()
        _ffi.check("ngpu_sim_param_rows", _ffi.lib().ngpu_sim_param_rows(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def classes(self) -> int:
        """Mechanism masks compiled into the kernel that runs this simulation
        (0: the ahead-of-time kernel, generic channel code); after init()."""
        n = C.c_int32()
        _ffi.check("ngpu_sim_classes", _ffi.lib().ngpu_sim_classes(self._h, C.byref(n)))
        return n.value

    def n_bad(self, stream=None) -> int:
        n = C.c_int32()
        _ffi.check("ngpu_sim_check", _ffi.lib().ngpu_sim_check(self._h, C.byref(n), _stream_ptr(stream)))
        return n.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            _ffi.lib().ngpu_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(cell: CellModel | Model, params, amps, dts, stim_node: int, stim_area_um2: float,
        rec_nodes, v_init: float, precision: str = "fp32") -> np.ndarray:
    """One complete simulation from host arrays through ``ngpu_run``.

    params [n_sets, n_params, n_sections]; amps [n_stim, nt] nA; dts [nt] ms.
    Returns V [n_sets, n_stim, n_rec, nt] (V before each step's update)."""
    model = cell if isinstance(cell, Model) else Model(cell)
    p = _as_f32(params)
    a = _as_f32(amps)
    nt = a.shape[1]
    d = _as_f32(np.broadcast_to(np.asarray(dts, dtype=np.float32), (nt,)))
    r = np.ascontiguousarray(np.asarray(rec_nodes, dtype=np.int32).reshape(-1))
    out = np.empty((p.shape[0], a.shape[0], r.size, nt), dtype=np.float32)
    _ffi.check("ngpu_run", _ffi.lib().ngpu_run(
        model.handle, p.shape[0], _ffi.ptr(p), a.shape[0], nt, _ffi.ptr(a), _ffi.ptr(d),
        int(stim_node), float(stim_area_um2), r.size, _ffi.ptr(r), float(v_init),
        _PREC[precision], _ffi.ptr(out)))
    return out


class Batch:
    """Several Simulators (different morphologies, one mechanism set and
    precision) advanced by single launches (ngpu_batch_*).  Each member
    keeps its own parameters, stimulus, recording and trace."""

    def __init__(self, sims: list[Simulator]):
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s._h for s in self.sims])
        h = C.c_void_p()
        _ffi.check("ngpu_batch_create", _ffi.lib().ngpu_batch_create(arr, len(self.sims), C.byref(h)))
        self._h = h

    def init(self, v_init: float, stream=None) -> None:
        _ffi.check("ngpu_batch_init", _ffi.lib().ngpu_batch_init(self._h, float(v_init), _stream_ptr(stream)))

    def advance(self, t0: int, n_steps: int, stream=None) -> None:
        _ffi.check("ngpu_batch_advance", _ffi.lib().ngpu_batch_advance(
            self._h, int(t0), int(n_steps), _stream_ptr(stream)))

    def run_graph(self, v_init: float, nt: int, chunk: int, stream) -> None:
        """init + every advance chunk as one CUDA graph on a non-default stream."""
        _ffi.check("ngpu_batch_run_graph", _ffi.lib().ngpu_batch_run_graph(
            self._h, float(v_init), int(nt), int(chunk), _stream_ptr(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _ffi.lib().ngpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
