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
    _dev: tuple | None = None

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

    # ---- the same on CUDA tensors: parameters, features and scores stay on the device
    def _tables(self):
        """(base parameters [P][S], free-parameter map [K][P][S], target
        features, feature spreads) as float64 CUDA tensors."""
        if self._dev is None:
            import torch
            w = np.zeros((self.n_params,) + self.base.shape)
            sec_region = np.array([self.cell.region_names[r] for r in self.cell.region])
            for j, (pname, regions) in enumerate(FREE12):
                w[j, MAINEN.param_index(pname), np.nonzero(np.isin(sec_region, regions))[0]] = 1.0
            t = [torch.tensor(np.asarray(x, dtype=np.float64), device="cuda")
                 for x in (self.base, w, self.target_f, self.scale)]
            self._dev = tuple(t)
        return self._dev

    def params_device(self, u):
        """params_of on the device: base x 2^u on each free parameter's
        sections, [n][P][S] float32."""
        import torch
        base, w, _, _ = self._tables()
        return (base[None] * torch.exp2(torch.einsum("nk,kps->nps", u.to(torch.float64), w))).float()

    def simulate_device(self, u, chunk_sets: int = 16384):
        """Features [n, n_stim, 20] (float32, on the device) of parameter
        vectors u [n, 12] (a CUDA tensor)."""
        import torch
        from .sim import Simulator
        t0 = time.perf_counter()
        out = []
        for i in range(0, u.shape[0], chunk_sets):
            uu = u[i:i + chunk_sets]
            sim = Simulator(self.cell, uu.shape[0], self.n_stim, "fp32")
            sim.set_params(self.params_device(uu))
            sim.set_stimulus(self.amps, np.full(self.amps.shape[1], self.dt, np.float32), 0, float(self.cell.area[0]))
            sim.set_recording(np.array([0], dtype=np.int32), self.rec_every)
            sim.init(-70.0)
            sim.advance(0, self.amps.shape[1])
            out.append(sim.features(self.dt * self.rec_every, self.stim_on, self.stim_off))
            sim.close()
        self.sim_count += u.shape[0]
        self.sim_seconds += time.perf_counter() - t0
        return torch.cat(out)

    def score_device(self, f):
        _, _, target, scale = self._tables()
        d = (f.to(target.dtype) - target[None]) / scale[None, None, :]
        return (d * d).mean(dim=(1, 2))

    def objectives_device(self, f):
        """One objective per (protocol, feature): |difference| in units of the
        feature's spread, [n][n_stim * 20]."""
        _, _, target, scale = self._tables()
        d = (f.to(target.dtype) - target[None]) / scale[None, None, :]
        return d.abs().reshape(d.shape[0], -1)


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


def run_device(prob: FitProblem, pop_size: int, generations: int, seed: int = 0,
               selector: str = "truncation") -> GAResult:
    """The GA with every step on the device (csrc/ga.cuh): offspring by the
    variation kernel, parameters expanded, simulated and reduced to features
    and scores without a host copy, survivors by (mu + lambda) truncation on
    the scalar score or by NSGA-II on the per-(protocol, feature)
    objectives.  The host reads one number per generation (the best score,
    for the result)."""
    import torch

    from .ga_device import DeviceGA, select_nsga2, select_truncation
    if selector not in ("truncation", "nsga2"):
        raise ValueError("selector: 'truncation' or 'nsga2'")
    ga = DeviceGA(prob.n_params, seed=seed)
    res = GAResult()
    t0 = time.perf_counter()
    gen = torch.Generator(device="cuda").manual_seed(seed)
    pop = torch.rand((pop_size, prob.n_params), generator=gen, device="cuda", dtype=torch.float64) * 2.0 - 1.0
    f = prob.simulate_device(pop)
    score = prob.score_device(f)
    if selector == "nsga2":
        obj = prob.objectives_device(f)
        _, rank, crowd, _ = select_nsga2(obj, pop_size)
    else:
        rank = torch.zeros(pop_size, dtype=torch.int32, device="cuda")
        crowd = -score
    for g in range(generations):
        kids = ga.offspring(pop, rank, crowd, pop_size, g)
        fk = prob.simulate_device(kids)
        allp, alls = torch.cat([pop, kids]), torch.cat([score, prob.score_device(fk)])
        if selector == "nsga2":
            allo = torch.cat([obj, prob.objectives_device(fk)])
            idx, rk, cr, _ = select_nsga2(allo, pop_size)
            pop, score, obj, rank, crowd = allp[idx], alls[idx], allo[idx], rk[idx], cr[idx]
        else:
            idx = select_truncation(alls, pop_size)
            pop, score = allp[idx], alls[idx]
            crowd = -score
        res.best.append(float(score.min()))
        res.time.append(time.perf_counter() - t0)
        res.sims.append(prob.sim_count)
    res.best_u = pop[int(torch.argmin(score))].cpu().numpy()
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


# ------------------------------------------- surrogate trained once, screened GA on the device
def inputs_device(u, n_stim: int):
    """_inputs on the device: (parameters, protocol one-hot) rows [n * n_stim, 12 + n_stim] float32 for
    u [n, 12] (a CUDA tensor)."""
    import torch
    n, k = u.shape
    x = torch.zeros((n * n_stim, k + n_stim), dtype=torch.float32, device=u.device)
    x[:, :k] = u.float().repeat_interleave(n_stim, dim=0)
    x[torch.arange(n * n_stim, device=u.device), k + torch.arange(n_stim, device=u.device).repeat(n)] = 1.0
    return x


@dataclass
class SurrogateFit:
    net: object
    n_train: int          # simulated parameter sets (each over every protocol)
    sim_seconds: float    # wall time of the training simulations
    train_seconds: float  # wall time of the network's training
    final_loss: float


def train_surrogate(prob: FitProblem, n_train: int = 200_000, epochs: int = 30, batch: int = 4096,
                    lr: float = 1e-3, seed: int = 0) -> SurrogateFit:
    """The surrogate of prob's cell and protocols: n_train parameter sets
    drawn uniformly over the whole search space (independent of any fit's
    target, so one network serves every fit of this cell), simulated on the
    device, features kept in HBM, and the network trained on them with its
    own BF16 tensor-core kernels."""
    import torch

    from .surrogate import SurrogateMLP
    gen = torch.Generator(device="cuda").manual_seed(seed)
    t0 = time.perf_counter()
    u = torch.rand((n_train, prob.n_params), generator=gen, device="cuda", dtype=torch.float64) * 2.0 - 1.0
    f = prob.simulate_device(u)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = SurrogateMLP(prob.n_params + prob.n_stim, features.N_FEATURES, seed=seed, lr=lr)
    hist = net.train(inputs_device(u, prob.n_stim), f.reshape(-1, f.shape[-1]).float(), epochs=epochs, batch=batch,
                     lr=lr, seed=seed)
    torch.cuda.synchronize()
    return SurrogateFit(net, n_train, t1 - t0, time.perf_counter() - t1, float(hist[-1]) if hist else float("nan"))


def run_screened_device(prob: FitProblem, net, pop_size: int, generations: int, keep_frac: float = 0.1,
                        err_bound: float = 0.5, tune_epochs: int = 1, seed: int = 0, target: float | None = None,
                        time_budget: float | None = None) -> GAResult:
    """The surrogate-screened GA with a trained network, every step on the
    device: offspring by the variation kernel (csrc/ga.cuh), the network's
    predicted features and scores for all of them, the best-predicted
    keep_frac simulated, (mu + lambda) truncation among simulated
    individuals.  Every generation the network's error on the simulated
    individuals (mean |predicted - simulated| in units of each feature's
    spread) is measured; above err_bound that generation simulates every
    offspring instead (the plain GA's step).  The network is fine-tuned on
    each generation's simulations.  Stops after `generations`, once the best
    score is <= target, or once time_budget wall seconds have passed.  The
    host reads two numbers per generation (the error and the best score)."""
    import torch

    from .ga_device import DeviceGA, select_truncation
    ga = DeviceGA(prob.n_params, seed=seed)
    res = GAResult()
    t0 = time.perf_counter()
    gen = torch.Generator(device="cuda").manual_seed(seed)
    pop = torch.rand((pop_size, prob.n_params), generator=gen, device="cuda", dtype=torch.float64) * 2.0 - 1.0
    score = prob.score_device(prob.simulate_device(pop))
    rank = torch.zeros(pop_size, dtype=torch.int32, device="cuda")
    _, _, _, scale = prob._tables()
    n_keep = max(1, int(round(keep_frac * pop_size)))
    for g in range(generations):
        kids = ga.offspring(pop, rank, -score, pop_size, g)
        pred = net.predict(inputs_device(kids, prob.n_stim)).reshape(pop_size, prob.n_stim, -1)
        order = torch.argsort(prob.score_device(pred))
        chosen = kids[order[:n_keep]]
        fk = prob.simulate_device(chosen)
        err = float(((pred[order[:n_keep]].double() - fk.double()) / scale[None, None, :]).abs().mean())
        if err > err_bound:  # the network is off here: simulate every offspring
            rest = kids[order[n_keep:]]
            chosen, fk = torch.cat([chosen, rest]), torch.cat([fk, prob.simulate_device(rest)])
            res.notes.append((g, err, "fallback"))
        else:
            res.notes.append((g, err, "screened"))
        if tune_epochs > 0:
            net.train(inputs_device(chosen, prob.n_stim), fk.reshape(-1, fk.shape[-1]).float(), epochs=tune_epochs,
                      batch=4096, lr=3e-4, seed=seed + g + 1)
        allp, alls = torch.cat([pop, chosen]), torch.cat([score, prob.score_device(fk)])
        idx = select_truncation(alls, pop_size)
        pop, score = allp[idx], alls[idx]
        res.best.append(float(score[0]))
        res.time.append(time.perf_counter() - t0)
        res.sims.append(prob.sim_count)
        if (target is not None and res.best[-1] <= target) or (time_budget is not None and res.time[-1] >= time_budget):
            break
    res.best_u = pop[0].cpu().numpy()
    return res
