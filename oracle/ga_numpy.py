"""numpy restatement of the device genetic-algorithm steps
(neurogpu_b200/csrc/ga.cuh): the same counter-based random stream, the same
operators and the same orderings, to check the kernels against.

TEST INFRASTRUCTURE ONLY -- imported by tests/; never by the product.

Operators, from their publications:
  * SplitMix64 (Steele, Lea & Flood 2014) as the random stream: draw d of
    child c in generation g is splitmix64(key ^ splitmix64(c << 20 | d)),
    key = splitmix64(seed ^ splitmix64(g));
  * binary tournament on (front rank ascending, crowding descending), the
    first pick winning ties;
  * bounded simulated binary crossover (Deb & Agrawal), per-gene
    probability 1/2, and bounded polynomial mutation (Deb & Goyal);
  * (mu + lambda) truncation: a stable sort of the scores, NaN last;
  * NSGA-II (Deb, Pratap, Agarwal & Meyarivan 2002): fronts by peeling the
    non-dominated set, crowding distance per objective within each front
    (ends +inf, the others (f_next - f_prev) / (f_last - f_first), 0 for a
    flat front), summed over objectives in order; survivors sorted by
    (rank, -crowding, index).
Every sort breaks ties by index, as the kernels do.
"""
from __future__ import annotations

import numpy as np

U64 = np.uint64
DRAWS_FIXED = 6
DRAWS_PER_GENE = 5


def splitmix64(x):
    x = np.asarray(x, dtype=U64)
    with np.errstate(over="ignore"):
        x = x + U64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> U64(30))) * U64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> U64(27))) * U64(0x94D049BB133111EB)
    return x ^ (x >> U64(31))


def ga_key(seed: int, generation: int):
    return splitmix64(U64(seed) ^ splitmix64(U64(generation)))


def bits(key, child, d: int):
    ctr = (np.asarray(child, dtype=U64) << U64(20)) | U64(d)
    return splitmix64(key ^ splitmix64(ctr))


def uniform(key, child, d: int) -> np.ndarray:
    return (bits(key, child, d) >> U64(11)).astype(np.float64) * 2.0 ** -53


def index(key, child, d: int, n: int) -> np.ndarray:
    return (((bits(key, child, d) >> U64(32)) * U64(n)) >> U64(32)).astype(np.int64)


def _sbx_beta_q(beta, u, eta):
    alpha = 2.0 - beta ** -(eta + 1.0)
    return np.where(u <= 1.0 / alpha, (u * alpha) ** (1.0 / (eta + 1.0)),
                    (1.0 / (2.0 - u * alpha)) ** (1.0 / (eta + 1.0)))


def offspring(pop, rank, crowd, n_kids, low, up, eta_c, eta_m, cx_prob, p_mut, seed, generation):
    """Children [n_kids][n_genes] of pop [mu][n_genes]."""
    pop = np.asarray(pop, dtype=np.float64)
    mu, n_genes = pop.shape
    key = ga_key(seed, generation)
    ch = np.arange(n_kids, dtype=np.uint64)

    def tour(i, j):
        better = (rank[j] < rank[i]) | ((rank[j] == rank[i]) & (crowd[j] > crowd[i]))
        return np.where(better, j, i)
    p1 = tour(index(key, ch, 0, mu), index(key, ch, 1, mu))
    p2 = tour(index(key, ch, 2, mu), index(key, ch, 3, mu))
    mate = uniform(key, ch, 4) < cx_prob
    first = uniform(key, ch, 5) < 0.5
    span = up - low
    out = np.empty((n_kids, n_genes))
    with np.errstate(all="ignore"):
        for g in range(n_genes):
            d = DRAWS_FIXED + DRAWS_PER_GENE * g
            a, b = pop[p1, g], pop[p2, g]
            u_do, u, u_sw = uniform(key, ch, d), uniform(key, ch, d + 1), uniform(key, ch, d + 2)
            cross = (u_do < 0.5) & (np.abs(a - b) > 1e-14)
            x1, x2 = np.minimum(a, b), np.maximum(a, b)
            dx = x2 - x1
            y1 = np.clip(0.5 * (x1 + x2 - _sbx_beta_q(1.0 + 2.0 * (x1 - low) / dx, u, eta_c) * dx), low, up)
            y2 = np.clip(0.5 * (x1 + x2 + _sbx_beta_q(1.0 + 2.0 * (up - x2) / dx, u, eta_c) * dx), low, up)
            swap = u_sw < 0.5
            v = np.where(mate, np.where(cross, np.where(first != swap, y1, y2), np.where(first, a, b)), a)
            do_mut = uniform(key, ch, d + 3) < p_mut
            r = uniform(key, ch, d + 4)
            d1, d2 = (v - low) / span, (up - v) / span
            mp = 1.0 / (eta_m + 1.0)
            lo_val = 2.0 * r + (1.0 - 2.0 * r) * (1.0 - d1) ** (eta_m + 1.0)
            hi_val = 2.0 * (1.0 - r) + 2.0 * (r - 0.5) * (1.0 - d2) ** (eta_m + 1.0)
            dq = np.where(r < 0.5, lo_val ** mp - 1.0, 1.0 - hi_val ** mp)
            out[:, g] = np.where(do_mut, np.clip(v + dq * span, low, up), v)
    return out


def select_truncation(score, mu: int) -> np.ndarray:
    s = np.asarray(score, dtype=np.float64)
    key = np.where(np.isnan(s), np.inf, s)
    nan_last = np.isnan(s).astype(np.int64)
    return np.lexsort((np.arange(s.size), key, nan_last))[:mu]


def fronts(obj) -> np.ndarray:
    """Front rank of every row of obj [n][m] (NaN as +inf)."""
    f = np.where(np.isnan(obj), np.inf, np.asarray(obj, dtype=np.float64))
    n = f.shape[0]
    dom = np.zeros((n, n), dtype=bool)            # dom[i, j]: j dominates i
    for i0 in range(0, n, 256):
        fi = f[i0:i0 + 256, None, :]
        dom[i0:i0 + 256] = np.all(f[None] <= fi, axis=2) & np.any(f[None] < fi, axis=2)
    rank = np.full(n, -1, dtype=np.int64)
    remaining = np.ones(n, dtype=bool)
    front = 0
    while remaining.any():
        cur = remaining & ~np.any(dom & remaining[None, :], axis=1)
        rank[cur] = front
        remaining &= ~cur
        front += 1
    return rank


def crowding(obj, rank) -> np.ndarray:
    f = np.where(np.isnan(obj), np.inf, np.asarray(obj, dtype=np.float64))
    n, m = f.shape
    idx = np.arange(n)
    total = np.zeros(n)
    for k in range(m):
        order = np.lexsort((idx, f[:, k], rank))
        r = rank[order]
        fk = f[order, k]
        first = np.r_[True, r[1:] != r[:-1]]
        last = np.r_[r[1:] != r[:-1], True]
        start = np.maximum.accumulate(np.where(first, np.arange(n), 0))
        end = np.minimum.accumulate(np.where(last, np.arange(n), n)[::-1])[::-1]
        lo, hi = fk[start], fk[end]
        c = np.zeros(n)
        inner = ~(first | last)
        with np.errstate(all="ignore"):
            span = hi - lo
            val = (np.r_[fk[1:], 0.0] - np.r_[0.0, fk[:-1]]) / span
        c[inner] = np.where(hi[inner] == lo[inner], 0.0, val[inner])
        c[first | last] = np.inf
        contrib = np.empty(n)
        contrib[order] = c
        total = total + contrib
    return total


def select_nsga2(obj, mu: int):
    """(survivors [mu], rank [n], crowding [n], number of fronts)."""
    rank = fronts(obj)
    crowd = crowding(obj, rank)
    order = np.lexsort((np.arange(rank.size), -crowd, rank))
    return order[:mu], rank, crowd, int(rank.max()) + 1
