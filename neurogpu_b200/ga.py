"""Genetic algorithm around the simulator, plain and surrogate-screened.

The reference's GA (GUI/DEAP_helper.py:131-271 with DEAP's varOr /
eaMuPlusLambda, bluepyopt's settings in P/optimize_parameters_genetic_alg.py)
evaluates every offspring by simulating it.  Here the operators are restated
vectorised over the whole population (numpy): binary tournament selection,
simulated binary crossover and polynomial mutation within bounds (DEAP's
cxSimulatedBinaryBounded / mutPolynomialBounded, Deb's published
formulas), (mu + lambda) truncation selection.

The screened GA generates the same offspring, lets the surrogate network
predict their features, simulates only the best-predicted fraction and
selects among simulated individuals only.  Every generation it measures the
surrogate's error on the individuals it simulated; above `err_bound` (mean
absolute error in units of each feature's spread) that generation falls back
to simulating every offspring, and the surrogate is fine-tuned on all
simulated data so far.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import configs, features
from .mechsets import MAINEN

# the 12 fitted parameters: 8 conductances and 4 rate constants, as log2
# multipliers in [-1, 1] of their nominal values
FREE12 = configs.MAINEN_FREE + (("Ra_km", ("soma", "dend")), ("Ra_kv", ("soma", "axon")),
                                 ("Ra_na", ("soma", "dend", "axon")), ("Rd_na", ("soma", "dend", "axon")))


@dataclass
class FitProblem:
    """Fit 12 parameters of an HH-type cell to a target's features over a
    few step-current protocols."""
    n_comp: int = 500
    t_stop: float = 500.0
    dt: float = 0.025
    stim_on: float = 50.0
    stim_off: float = 450.0
    levels: tuple = (0.2, 0.5, 1.0)
    rec_every: int = 10
    seed: int = 5
    target_u: np.ndarray | None = None
    cell: object = None
    base: np.ndarray = None
    target_f: np.ndarray = None
    scale: np.ndarray = None
    sim_count: int = 0
    sim_seconds: float = 0.0

    def __post_init__(self):
        rng = np.random.default_rng(self.seed)
        secs = configs.hh_morphology(rng, self.n_comp)
        self.cell = configs.build_model(secs, MAINEN, configs.MAINEN_REGIONS, configs.MAINEN_MECHS, ra=150.0,
                                        cm_of_region={"soma": 0.75, "dend": 1.5, "axon": 0.75})
        self.base = configs._region_params(self.cell, MAINEN, configs.MAINEN_NOMINAL, configs.MAINEN_FIXED)
        nt = int(round(self.t_stop / self.dt))
        self.amps = configs.step_amps(self.levels, nt, self.dt, self.stim_on, self.stim_off)
        if self.target_u is None:
            self.target_u = rng.uniform(-0.8, 0.8, len(FREE12))
        self.target_f = self.simulate(self.target_u[None, :])[0]
        probe = self.simulate(rng.uniform(-1, 1, (256, len(FREE12))))
        self.scale = probe.reshape(-1, probe.shape[-1]).std(0).clip(min=1e-3)
        self.sim_count = 0
        self.sim_seconds = 0.0

    @property
    def n_params(self) -> int:
        return len(FREE12)

    @property
    def n_stim(self) -> int:
        return len(self.levels)

    def params_of(self, u: np.ndarray) -> np.ndarray:
        return configs._apply_free(self.cell, MAINEN, self.base, FREE12, np.exp2(np.asarray(u, dtype=np.float64)))

    def simulate(self, u: np.ndarray, chunk_sets: int = 16384) -> np.ndarray:
        """Features [n, n_stim, 20] of parameter vectors u [n, 12]."""
        import torch
        from .sim import Simulator
        t0 = time.perf_counter()
        out = []
        for i in range(0, len(u), chunk_sets):
            uu = np.asarray(u[i:i + chunk_sets])
            sim = Simulator(self.cell, len(uu), self.n_stim, "fp32")
            sim.set_params(self.params_of(uu))
            sim.set_stimulus(self.amps, np.full(self.amps.shape[1], self.dt, np.float32), 0, float(self.cell.area[0]))
            sim.set_recording(np.array([0], dtype=np.int32), self.rec_every)
            sim.init(-70.0)
            sim.advance(0, self.amps.shape[1])
            # features where the trace lies (ngpu_sim_features): traces are never copied
            f = sim.features(self.dt * self.rec_every, self.stim_on, self.stim_off)
            out.append(f.cpu().numpy())
            sim.close()
        torch.cuda.synchronize()
        self.sim_count += len(u)
        self.sim_seconds += time.perf_counter() - t0
        return np.concatenate(out).astype(np.float64)

    def score(self, f: np.ndarray) -> np.ndarray:
        """Mean squared feature difference to the target in units of each
        feature's spread, over protocols and features: [n]."""
        d = (np.asarray(f) - self.target_f[None]) / self.scale[None, None, :]
        return np.mean(d * d, axis=(1, 2))


# ------------------------------------------------------------------ operators
def tournament(rng, score, k, size=2):
    idx = rng.integers(0, len(score), (k, size))
    return idx[np.arange(k), np.argmin(score[idx], axis=1)]


def sbx(rng, a, b, eta=10.0, low=-1.0, up=1.0, p_gene=0.5):
    """Bounded simulated binary crossover of parent rows a, b (Deb & Agrawal)."""
    c1, c2 = a.copy(), b.copy()
    do = (rng.random(a.shape) < p_gene) & (np.abs(a - b) > 1e-14)
    x1, x2 = np.minimum(a, b), np.maximum(a, b)
    rand = rng.random(a.shape)
    with np.errstate(all="ignore"):
        def child(beta_edge):
            alpha = 2.0 - beta_edge ** -(eta + 1)
            beta_q = np.where(rand <= 1.0 / alpha, (rand * alpha) ** (1.0 / (eta + 1)),
                              (1.0 / (2.0 - rand * alpha)) ** (1.0 / (eta + 1)))
            return beta_q
        bq1 = child(1.0 + 2.0 * (x1 - low) / (x2 - x1))
        bq2 = child(1.0 + 2.0 * (up - x2) / (x2 - x1))
        y1 = np.clip(0.5 * (x1 + x2 - bq1 * (x2 - x1)), low, up)
        y2 = np.clip(0.5 * (x1 + x2 + bq2 * (x2 - x1)), low, up)
    swap = rng.random(a.shape) < 0.5
    c1 = np.where(do, np.where(swap, y2, y1), c1)
    c2 = np.where(do, np.where(swap, y1, y2), c2)
    return c1, c2


def poly_mutate(rng, x, eta=20.0, low=-1.0, up=1.0, p_gene=None):
    """Bounded polynomial mutation (Deb & Goyal)."""
    p_gene = 1.0 / x.shape[1] if p_gene is None else p_gene
    do = rng.random(x.shape) < p_gene
    d1, d2 = (x - low) / (up - low), (up - x) / (up - low)
    r = rng.random(x.shape)
    mp = 1.0 / (eta + 1.0)
    xy = np.where(r < 0.5, 1.0 - d1, 1.0 - d2)
    val = np.where(r < 0.5, 2.0 * r + (1.0 - 2.0 * r) * xy ** (eta + 1), 2.0 * (1.0 - r) + 2.0 * (r - 0.5) * xy ** (eta + 1))
    dq = np.where(r < 0.5, val ** mp - 1.0, 1.0 - val ** mp)
    return np.where(do, np.clip(x + dq * (up - low), low, up), x)


def offspring(rng, pop, score, n, cx_prob=0.9):
    i, j = tournament(rng, score, n), tournament(rng, score, n)
    a, b = pop[i], pop[j]
    c1, c2 = sbx(rng, a, b)
    mate = rng.random(n) < cx_prob
    kids = np.where(mate[:, None], np.where(rng.random(n)[:, None] < 0.5, c1, c2), a)
    return poly_mutate(rng, kids)


@dataclass
class GAResult:
    best: list = field(default_factory=list)        # best score after each generation
    time: list = field(default_factory=list)        # wall seconds at the end of each generation
    sims: list = field(default_factory=list)        # simulations so far
    notes: list = field(default_factory=list)
    best_u: np.ndarray | None = None

    def time_to(self, target: float) -> float | None:
        for b, t in zip(self.best, self.time):
            if b <= target:
                return t
        return None


def run_plain(prob: FitProblem, pop_size: int, generations: int, seed: int = 0) -> GAResult:
    rng = np.random.default_rng(seed)
    res = GAResult()
    t0 = time.perf_counter()
    pop = rng.uniform(-1, 1, (pop_size, prob.n_params))
    score = prob.score(prob.simulate(pop))
    for g in range(generations):
        kids = offspring(rng, pop, score, pop_size)
        ks = prob.score(prob.simulate(kids))
        allp, alls = np.concatenate([pop, kids]), np.concatenate([score, ks])
        keep = np.argsort(alls)[:pop_size]
        pop, score = allp[keep], alls[keep]
        res.best.append(float(score[0]))
        res.time.append(time.perf_counter() - t0)
        res.sims.append(prob.sim_count)
    res.best_u = pop[0]
    return res


def _inputs(u: np.ndarray, n_stim: int) -> np.ndarray:
    """(parameters, protocol one-hot) rows for every (individual, protocol)."""
    n = len(u)
    x = np.zeros((n * n_stim, u.shape[1] + n_stim), dtype=np.float32)
    x[:, :u.shape[1]] = np.repeat(u, n_stim, axis=0)
    x[np.arange(n * n_stim), u.shape[1] + np.tile(np.arange(n_stim), n)] = 1.0
    return x


def run_screened(prob: FitProblem, pop_size: int, generations: int, keep_frac: float = 0.1,
                 n_train: int = 20000, train_epochs: int = 30, tune_epochs: int = 3, err_bound: float = 0.5,
                 seed: int = 0, target: float | None = None, time_budget: float | None = None) -> GAResult:
    """The surrogate-screened GA (wall time includes building the training
    set and training).  Stops after `generations`, or once the best score is
    <= target, or once time_budget wall seconds have passed."""
    from .surrogate import SurrogateMLP
    rng = np.random.default_rng(seed)
    res = GAResult()
    t0 = time.perf_counter()
    pop = rng.uniform(-1, 1, (pop_size, prob.n_params))
    extra = rng.uniform(-1, 1, (max(0, n_train - pop_size), prob.n_params))
    f_all = prob.simulate(np.concatenate([pop, extra]))
    score = prob.score(f_all[:pop_size])
    U, F = np.concatenate([pop, extra]), f_all
    net = SurrogateMLP(prob.n_params + prob.n_stim, features.N_FEATURES, seed=seed)
    X, Y = _inputs(U, prob.n_stim), F.reshape(-1, F.shape[-1]).astype(np.float32)
    net.train(X, Y, epochs=train_epochs, batch=4096, lr=1e-3, seed=seed)
    n_keep = max(1, int(round(keep_frac * pop_size)))
    for g in range(generations):
        kids = offspring(rng, pop, score, pop_size)
        pred = net.predict(_inputs(kids, prob.n_stim)).cpu().numpy().reshape(pop_size, prob.n_stim, -1)
        order = np.argsort(prob.score(pred))
        chosen = kids[order[:n_keep]]
        fk = prob.simulate(chosen)
        err = float(np.mean(np.abs((pred[order[:n_keep]] - fk) / prob.scale[None, None, :])))
        if err > err_bound:                          # the surrogate is off: simulate every offspring
            rest = kids[order[n_keep:]]
            fr = prob.simulate(rest)
            chosen, fk = np.concatenate([chosen, rest]), np.concatenate([fk, fr])
            res.notes.append((g, err, "fallback"))
        else:
            res.notes.append((g, err, "screened"))
        U, F = np.concatenate([U, chosen]), np.concatenate([F, fk])
        X, Y = _inputs(U, prob.n_stim), F.reshape(-1, F.shape[-1]).astype(np.float32)
        net.train(X[-len(chosen) * prob.n_stim * 8:], Y[-len(chosen) * prob.n_stim * 8:], epochs=tune_epochs,
                  batch=4096, lr=3e-4, seed=seed + g + 1)
        ks = prob.score(fk)
        allp, alls = np.concatenate([pop, chosen]), np.concatenate([score, ks])
        keep = np.argsort(alls)[:pop_size]
        pop, score = allp[keep], alls[keep]
        res.best.append(float(score[0]))
        res.time.append(time.perf_counter() - t0)
        res.sims.append(prob.sim_count)
        if (target is not None and score[0] <= target) or (time_budget is not None and res.time[-1] >= time_budget):
            break
    res.best_u = pop[0]
    return res
