"""Genetic-algorithm steps on the GPU (ngpu_ga_* in include/ngpu.h):
offspring, (mu + lambda) truncation and NSGA-II selection on CUDA tensors,
so that a generation's population, children, features and scores stay in
device memory.

The reference runs DEAP's operators on the host between simulator calls
(GUI/DEAP_helper.py:126-271; bluepyopt's DEAPOptimisation at
Figures/Figure4_DEAP/optimize_parameters_genetic_alg.py:49, eta 20,
crossover 0.7, mutation 0.3).  The kernels (csrc/ga.cuh) restate the
published operators: tournament, bounded SBX, bounded polynomial mutation,
truncation, non-dominated sorting and crowding distance.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _ffi


def _stream(stream) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev(t: torch.Tensor, dtype: torch.dtype, name: str) -> torch.Tensor:
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError(f"{name} must be a CUDA tensor")
    return t.to(dtype).contiguous()


class DeviceGA:
    """Variation operators of one GA run: genes in [low, up], SBX spread
    eta_c, mutation spread eta_m, crossover probability cx_prob, per-gene
    mutation probability p_mut (default 1 / n_genes), random stream seed."""

    def __init__(self, n_genes: int, low: float = -1.0, up: float = 1.0, eta_c: float = 10.0, eta_m: float = 20.0,
                 cx_prob: float = 0.9, p_mut: float | None = None, seed: int = 0):
        self.n_genes = int(n_genes)
        self.low, self.up = float(low), float(up)
        self.eta_c, self.eta_m = float(eta_c), float(eta_m)
        self.cx_prob = float(cx_prob)
        self.p_mut = 1.0 / n_genes if p_mut is None else float(p_mut)
        self.seed = int(seed)

    def offspring(self, pop: torch.Tensor, rank: torch.Tensor, crowd: torch.Tensor, n_kids: int, generation: int,
                  stream=None) -> torch.Tensor:
        """Children [n_kids][n_genes] (float64) of pop [mu][n_genes]; parents
        win tournaments by lower rank, then higher crowd."""
        pop = _dev(pop, torch.float64, "pop")
        mu = pop.shape[0]
        if pop.ndim != 2 or pop.shape[1] != self.n_genes:
            raise ValueError(f"pop must be [mu][{self.n_genes}]")
        rank = _dev(rank, torch.int32, "rank")
        crowd = _dev(crowd, torch.float64, "crowd")
        if rank.numel() != mu or crowd.numel() != mu:
            raise ValueError("rank and crowd need one entry per individual")
        kids = torch.empty((n_kids, self.n_genes), dtype=torch.float64, device=pop.device)
        _ffi.check("ngpu_ga_offspring", _ffi.lib().ngpu_ga_offspring(
            C.c_void_p(pop.data_ptr()), C.c_void_p(rank.data_ptr()), C.c_void_p(crowd.data_ptr()), mu,
            self.n_genes, int(n_kids), self.low, self.up, self.eta_c, self.eta_m, self.cx_prob, self.p_mut,
            self.seed & (2 ** 64 - 1), int(generation), C.c_void_p(kids.data_ptr()), _stream(stream)))
        return kids


def select_truncation(score: torch.Tensor, mu: int, stream=None) -> torch.Tensor:
    """Indices (int64) of the mu smallest scores, best first (NaN last, ties
    by index)."""
    s = _dev(score, torch.float64, "score")
    out = torch.empty(mu, dtype=torch.int32, device=s.device)
    _ffi.check("ngpu_ga_select_truncation", _ffi.lib().ngpu_ga_select_truncation(
        C.c_void_p(s.data_ptr()), s.numel(), int(mu), C.c_void_p(out.data_ptr()), _stream(stream)))
    return out.long()


def select_nsga2(obj: torch.Tensor, mu: int, stream=None):
    """NSGA-II survivors of obj [n][m] (minimised): (indices [mu] in
    (rank, -crowd, index) order, rank [n] int32, crowd [n] float64, number
    of fronts as a 0-d int32 tensor on the device)."""
    f = _dev(obj, torch.float64, "obj")
    if f.ndim != 2:
        raise ValueError("obj must be [n][m]")
    n, m = f.shape
    out = torch.empty(mu, dtype=torch.int32, device=f.device)
    rank = torch.empty(n, dtype=torch.int32, device=f.device)
    crowd = torch.empty(n, dtype=torch.float64, device=f.device)
    nf = torch.empty((), dtype=torch.int32, device=f.device)
    _ffi.check("ngpu_ga_select_nsga2", _ffi.lib().ngpu_ga_select_nsga2(
        C.c_void_p(f.data_ptr()), n, m, int(mu), C.c_void_p(out.data_ptr()), C.c_void_p(rank.data_ptr()),
        C.c_void_p(crowd.data_ptr()), C.c_void_p(nf.data_ptr()), _stream(stream)))
    return out.long(), rank, crowd, nf
