"""The tree split of the simulation kernel (host side, no GPU needed).

The library reorders nodes heavy-first and cuts the tree at separator nodes
into work items: plain subtrees and segments (a heavy-path piece above a
lower separator plus its light subtrees).  ngpu_model_split_info exposes the
split; these tests check its invariants and replay the kernel's
S1 / S2 / S3 solve in numpy (one lane) against a dense solve of the same
tree matrix."""
import numpy as np
import pytest

from neurogpu_b200 import configs
from neurogpu_b200.mechsets import TTPC
from neurogpu_b200.model import CellModel, cable_coefficients
from neurogpu_b200.sim import Model


def _cells():
    out = {"passive128": configs.passive_cable(n_sets=1).cell,
           "hh500": configs.hh_active(n_sets=1).cell,
           "ttpc1501": configs.ttpc_like(n_sets=1).cell}
    rng = np.random.default_rng(5)
    # a pure chain, a star and a comb: the split's degenerate shapes
    comb = [-1] + [2 * ((i - 1) // 2) if i % 2 == 0 else (i - 2 if i > 2 else 0) for i in range(1, 81)]
    comb = np.array([-1] + [max(0, i - 2) if i % 2 else i - 1 for i in range(1, 81)], dtype=np.int32)
    for name, parent in (("chain64", np.arange(-1, 63, dtype=np.int32)),
                         ("star40", np.array([-1] + [0] * 39, dtype=np.int32)),
                         ("comb81", comb)):
        n = parent.size
        a, b, area = cable_coefficients(parent, np.full(n, 10.0), rng.uniform(1, 3, n), 100.0)
        mask = np.zeros((TTPC.n_mech, n), dtype=np.uint8)
        mask[TTPC.mech_index("pas")] = 1
        out[name] = CellModel(parent=parent, a=a, b=b, cm=np.ones(n), section=np.zeros(n, dtype=np.int32),
                              n_sections=1, mechset=TTPC, mech_mask=mask, area=area)
    return out


CELLS = _cells()
WARPS = [1, 2, 3, 4, 8]


def _internal(cell, info):
    """Parent / coefficients in the library's internal node order."""
    perm = info["perm"]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    par = np.array([-1] + [inv[cell.parent[perm[i]]] for i in range(1, perm.size)], dtype=np.int64)
    return par, cell.a[perm], cell.b[perm]


@pytest.mark.parametrize("name", list(CELLS))
@pytest.mark.parametrize("W", WARPS)
def test_split_invariants(ngpu_built, name, W):
    cell = CELLS[name]
    info = Model(cell).split_info(W)
    n = cell.n_nodes
    perm = info["perm"]
    assert sorted(perm) == list(range(n))
    par, _, _ = _internal(cell, info)
    assert par[0] == -1 and np.all(par[1:] < np.arange(1, n))       # still Hines order
    seps = info["seps"][:, 0]
    assert seps[0] == 0 and np.all(np.diff(seps) > 0)
    owner = np.full(n, -1)
    for k, (r, u, l, lk, lo, hi) in enumerate(info["comps"]):
        assert par[r] == u and u in seps
        nodes = list(range(lo, hi)) + (list(range(r, l)) if l >= 0 else [])
        if l >= 0:
            assert seps[lk] == l and par[l] == l - 1
            assert all(par[i] == i - 1 for i in range(r + 1, l))         # the spine is a path
        for i in nodes:
            assert owner[i] == -1
            owner[i] = k
    assert np.all((owner >= 0) != np.isin(np.arange(n), seps))        # items + separators cover all
    for k, (node, sp, seg) in enumerate(info["seps"]):
        if k == 0:
            continue
        if seg < 0:
            assert seps[sp] == par[node]
        else:
            c = info["comps"][seg]
            assert c[2] == node and seps[sp] == c[1]
    if W > 1:
        tot = n
        assert max((c[5] - c[4]) + (c[2] - c[0] if c[2] >= 0 else 0) for c in info["comps"]) <= tot


def _emulate(par, a, b, info, d, rhs, e):
    """The kernel's S1 / S2 / S3 solve for one lane, internal node order."""
    n = par.size
    js, ps = info["jslot"], info["pslot"]
    nj = max(1, js.max() + 1)
    jacc = np.zeros((nj, 2))
    row = np.zeros((n, 3))                       # scratch rows
    row[:, 0], row[:, 1], row[:, 2] = d, rhs, e
    sepv = np.zeros((max(1, len(info["seps"])), 4))
    jx = np.zeros(nj)

    def elim(i, carry):
        dd, rr = row[i, 0] + carry[0], row[i, 1] + carry[1]
        ei = row[i, 2]
        if js[i] >= 0:
            dd += jacc[js[i], 0]
            rr += jacc[js[i], 1]
            jacc[js[i]] = 0
        row[i, 0], row[i, 1] = rr / dd, a[i] / dd
        contrib = (-b[i] * row[i, 1], ei - b[i] * row[i, 0])
        if ps[i] < 0:
            return contrib
        jacc[ps[i]] += contrib
        return (0.0, 0.0)

    for (r, u, l, lk, lo, hi) in info["comps"]:           # S1
        carry = (0.0, 0.0)
        for i in range(hi - 1, lo - 1, -1):
            carry = elim(i, carry)
        if l >= 0:
            cd = cr = cw = 0.0
            for i in range(l - 1, r - 1, -1):
                dd, rr, ei = row[i, 0] + cd, row[i, 1] + cr, row[i, 2]
                if js[i] >= 0:
                    dd += jacc[js[i], 0]
                    rr += jacc[js[i], 1]
                    jacc[js[i]] = 0
                w = cw
                if i == l - 1:
                    w = -b[l]
                    rr += row[l, 2]
                row[i] = (rr / dd, a[i] / dd, w / dd)
                if i > r:
                    cd, cr, cw = -b[i] * row[i, 1], ei - b[i] * row[i, 0], -b[i] * row[i, 2]
                else:
                    jacc[ps[i]] += (-b[i] * row[i, 1], ei - b[i] * row[i, 0])
                    sepv[lk, 1] = b[i] * row[i, 2]
            al = be = ga = 0.0
            for i in range(r, l):
                rr_, cc, om = row[i]
                if i == r:
                    al, be, ga = -cc, om, rr_
                else:
                    al, be, ga = -cc * al, om - cc * be, rr_ - cc * ga
                row[i] = (ga, al, be)
            sepv[lk, 0], sepv[lk, 2], sepv[lk, 3] = a[l] * al, a[l] * be, -a[l] * ga
    seps = info["seps"]                                     # S2
    for k in range(len(seps) - 1, -1, -1):
        s, sp, seg = seps[k]
        dd = row[s, 0] + jacc[js[s], 0]
        rr = row[s, 1] + jacc[js[s], 1]
        jacc[js[s]] = 0
        A, B, eup = a[s], b[s], row[s, 2]
        if seg >= 0:
            A, B = sepv[k, 0], sepv[k, 1]
            dd += sepv[k, 2]
            rr += sepv[k, 3]
            eup = 0.0
        if k == 0:
            row[s, 0] = rr / dd
            break
        row[s, 0], row[s, 1] = rr / dd, A / dd
        jacc[js[seps[sp, 0]]] += (-B * row[s, 1], eup - B * row[s, 0])
    x = np.zeros(n)
    for k, (s, sp, seg) in enumerate(seps):
        x[s] = row[s, 0] if k == 0 else row[s, 0] - row[s, 1] * jx[js[seps[sp, 0]]]
        jx[js[s]] = x[s]
    for (r, u, l, lk, lo, hi) in info["comps"]:             # S3
        if l >= 0:
            for i in range(r, l):
                x[i] = row[i, 0] + row[i, 1] * jx[js[u]] + row[i, 2] * jx[js[l]]
                if js[i] >= 0:
                    jx[js[i]] = x[i]
        xprev = 0.0
        for i in range(lo, hi):
            xp = xprev if ps[i] < 0 else jx[ps[i]]
            x[i] = row[i, 0] - row[i, 1] * xp
            if js[i] >= 0:
                jx[js[i]] = x[i]
            xprev = x[i]
    return x


@pytest.mark.parametrize("name", list(CELLS))
@pytest.mark.parametrize("W", WARPS)
def test_split_solve_matches_dense(ngpu_built, name, W):
    cell = CELLS[name]
    info = Model(cell).split_info(W)
    par, a, b = _internal(cell, info)
    n = cell.n_nodes
    rng = np.random.default_rng(W * 1000 + n)
    dconst = -a.copy()
    dconst[0] = 0.0
    np.add.at(dconst, par[1:], -b[1:])
    d = rng.uniform(0.01, 2.0, n) + 0.04 + dconst
    rhs = rng.normal(0, 1, n)
    e = rng.normal(0, 0.1, n)
    e[0] = 0.0
    x = _emulate(par, a, b, info, d, rhs, e)
    # dense: row i: d_i x_i + a_i x_p + sum_c b_c x_c = rhs_i + sum_c e_c
    A = np.diag(d)
    bvec = rhs.copy()
    for i in range(1, n):
        p = par[i]
        A[i, p] += a[i]
        A[p, i] += b[i]
        bvec[p] += e[i]
    np.testing.assert_allclose(x, np.linalg.solve(A, bvec), rtol=1e-9, atol=1e-11)


def test_ttpc_split_is_balanced(ngpu_built):
    """The 1501-node pyramidal tree splits into items no larger than ~1/W of
    the work and a skeleton of a few dozen separators."""
    cell = CELLS["ttpc1501"]
    info = Model(cell).split_info(8)
    sizes = [(c[5] - c[4]) + (c[2] - c[0] if c[2] >= 0 else 0) for c in info["comps"]]
    assert len(info["seps"]) <= 64
    assert max(sizes) <= 0.25 * cell.n_nodes
