"""The tree split of the simulation kernel (host side, no GPU needed).

ngpu_model_partition exposes the split the kernel uses: a top tree solved by
warp 0 and subtrees owned by single warps.  These tests check its invariants
and replay the kernel's three-phase elimination / back-substitution in numpy
(one lane) against a dense solve of the same tree matrix."""
import numpy as np
import pytest

from neurogpu_b200 import configs
from neurogpu_b200.model import CellModel, random_binary_cable, cable_coefficients
from neurogpu_b200.mechsets import TTPC
from neurogpu_b200.sim import Model


def _cells():
    out = {"passive128": configs.passive_cable(n_sets=1).cell,
           "hh500": configs.hh_active(n_sets=1).cell,
           "ttpc1501": configs.ttpc_like(n_sets=1).cell}
    rng = np.random.default_rng(5)
    # a pure chain and a star: the split's degenerate shapes
    for name, parent in (("chain64", np.arange(-1, 63, dtype=np.int32)),
                         ("star40", np.array([-1] + [0] * 39, dtype=np.int32))):
        n = parent.size
        a, b, area = cable_coefficients(parent, np.full(n, 10.0), rng.uniform(1, 3, n), 100.0)
        mask = np.zeros((TTPC.n_mech, n), dtype=np.uint8)
        mask[TTPC.mech_index("pas")] = 1
        out[name] = CellModel(parent=parent, a=a, b=b, cm=np.ones(n), section=np.zeros(n, dtype=np.int32),
                              n_sections=1, mechset=TTPC, mech_mask=mask, area=area)
    return out


CELLS = _cells()


def _runs(mask_nodes):
    """Maximal runs of consecutive node indices."""
    idx = np.nonzero(mask_nodes)[0]
    if idx.size == 0:
        return []
    cuts = np.nonzero(np.diff(idx) != 1)[0]
    starts = np.concatenate([[idx[0]], idx[cuts + 1]])
    ends = np.concatenate([idx[cuts] + 1, [idx[-1] + 1]])
    return list(zip(starts, ends))


@pytest.mark.parametrize("name", list(CELLS))
@pytest.mark.parametrize("W", [1, 2, 4, 8, 16])
def test_split_invariants(ngpu_built, name, W):
    cell = CELLS[name]
    part = Model(cell).partition(W)
    top, owner, parent = part["top"], part["owner"], cell.parent
    n = cell.n_nodes
    assert top[0]
    assert np.all((owner >= 0) != top)                  # every node: top xor owned
    assert np.all(owner < W)
    for i in range(1, n):
        if top[i]:
            assert top[parent[i]]                          # top tree is connected
        elif not top[parent[i]]:
            assert owner[i] == owner[parent[i]]            # a subtree stays on one warp
    for i in range(1, n):                                  # far children and subtree roots
        far = parent[i] != i - 1 or (not top[i] and top[parent[i]])
        assert (part["pslot"][i] >= 0) == far
        if far:
            assert part["pslot"][i] == part["jslot"][parent[i]]


def _emulate(cell, part, d, rhs, e):
    """The kernel's S1 / S2 / S3 solve for one lane."""
    a, b, parent = cell.a, cell.b, cell.parent
    js, ps, top, owner = part["jslot"], part["pslot"], part["top"], part["owner"]
    n = cell.n_nodes
    jacc = np.zeros((max(1, part["n_jslots"]), 2))
    r = np.zeros(n)
    c = np.zeros(n)

    def elim(i, cd_cr):
        dd, rr = d[i] + cd_cr[0], rhs[i] + cd_cr[1]
        if js[i] >= 0:
            dd += jacc[js[i], 0]
            rr += jacc[js[i], 1]
            jacc[js[i]] = 0
        if i == 0:
            r[0], c[0] = rr / dd, 0.0
            return (0.0, 0.0)
        r[i], c[i] = rr / dd, a[i] / dd
        contrib = (-b[i] * c[i], e[i] - b[i] * r[i])
        if ps[i] < 0:
            return contrib
        jacc[ps[i]] += contrib
        return (0.0, 0.0)

    for w in range(owner.max() + 1 if (owner >= 0).any() else 0):   # S1
        for lo, hi in reversed(_runs(owner == w)):
            carry = (0.0, 0.0)
            for i in range(hi - 1, lo - 1, -1):
                carry = elim(i, carry)
    carry = (0.0, 0.0)                                               # S2
    tops = np.nonzero(top)[0]
    for i in tops[::-1]:
        carry = elim(i, carry)
    x = np.zeros(n)
    jx = np.zeros(max(1, part["n_jslots"]))

    def back(i, xprev):
        xp = 0.0 if i == 0 else (xprev if ps[i] < 0 else jx[ps[i]])
        x[i] = r[i] - c[i] * xp
        if js[i] >= 0:
            jx[js[i]] = x[i]
        return x[i]

    xprev = 0.0
    for i in tops:
        xprev = back(i, xprev)
    for w in range(owner.max() + 1 if (owner >= 0).any() else 0):   # S3
        for lo, hi in _runs(owner == w):
            xprev = 0.0
            for i in range(lo, hi):
                xprev = back(i, xprev)
    return x


@pytest.mark.parametrize("name", list(CELLS))
@pytest.mark.parametrize("W", [1, 3, 8])
def test_split_solve_matches_dense(ngpu_built, name, W):
    cell = CELLS[name]
    part = Model(cell).partition(W)
    n = cell.n_nodes
    rng = np.random.default_rng(W * 1000 + n)
    g = rng.uniform(0.01, 2.0, n)
    dconst = -cell.a.copy()
    dconst[0] = 0.0
    np.add.at(dconst, cell.parent[1:], -cell.b[1:])
    d = g + 0.04 + dconst
    rhs = rng.normal(0, 1, n)
    e = rng.normal(0, 0.1, n)
    e[0] = 0.0
    x = _emulate(cell, part, d, rhs, e)
    # dense: row i: d_i x_i + a_i x_p + sum_c b_c x_c = rhs_i + sum_c e_c
    A = np.diag(d)
    bvec = rhs.copy()
    for i in range(1, n):
        p = cell.parent[i]
        A[i, p] += cell.a[i]
        A[p, i] += cell.b[i]
        bvec[p] += e[i]
    np.testing.assert_allclose(x, np.linalg.solve(A, bvec), rtol=1e-10, atol=1e-12)
