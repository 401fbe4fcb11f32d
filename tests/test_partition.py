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
# CTA warps of the lane-instance layout; 16 and 32 split the tree into the
# 32 and 64 items of the warp-instance layout
WARPS = [1, 2, 3, 4, 8, 16, 32]


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
    if W > 1 and len(info["comps"]):  # (a split finer than the tree leaves separators only)
        tot = n
        assert max((c[5] - c[4]) + (c[2] - c[0] if c[2] >= 0 else 0) for c in info["comps"]) <= tot


def _emulate(par, a, b, info, ex_own, rhs, e, dtype=np.float64):
    """The kernel's S1 / S2 / S3 solve for one lane, internal node order, in
    the kernel's excess form: each row carries its excess (row sum: g +
    cm/dt plus what eliminated children leak to ground) instead of its full
    diagonal, which is rebuilt as excess + |couplings still in the row| when
    the row is eliminated.  dtype float32 mimics the FP32 kernel, including
    its FP64 junction sums."""
    R = dtype
    n = par.size
    a = a.astype(R)
    b = b.astype(R)
    js, ps = info["jslot"], info["pslot"]
    nj = max(1, js.max() + 1)
    jacc = np.zeros((nj, 2))                     # FP64 (excess, rhs)
    row = np.zeros((n, 3), dtype=R)              # scratch rows
    row[:, 0], row[:, 1], row[:, 2] = ex_own, rhs, e
    sepv = np.zeros((max(1, len(info["seps"])), 4), dtype=R)
    jx = np.zeros(nj, dtype=R)
    one = R(1)

    def take(i, cx, cr):
        if js[i] >= 0:
            x = R(np.float64(row[i, 0]) + np.float64(cx) + jacc[js[i], 0])
            r = R(np.float64(row[i, 1]) + np.float64(cr) + jacc[js[i], 1])
            jacc[js[i]] = 0
            return x, r
        return R(row[i, 0] + cx), R(row[i, 1] + cr)

    def elim(i, carry):
        ex, rr = take(i, *carry)
        ei = row[i, 2]
        if i == 0:
            row[0, 0], row[0, 1] = rr / ex, 0
            return (R(0), R(0))
        inv = one / R(ex - a[i])
        row[i, 0], row[i, 1] = rr * inv, a[i] * inv
        contrib = (R(-b[i] * (ex * inv)), R(ei - b[i] * row[i, 0]))
        if ps[i] < 0:
            return contrib
        jacc[ps[i]] += np.float64(contrib[0]), np.float64(contrib[1])
        return (R(0), R(0))

    for (r, u, l, lk, lo, hi) in info["comps"]:           # S1
        carry = (R(0), R(0))
        for i in range(hi - 1, lo - 1, -1):
            carry = elim(i, carry)
        if l >= 0:
            cx = cr = cw = R(0)
            P, Gs, Bs, Ds = one, R(0), R(0), R(0)
            for i in range(l - 1, r - 1, -1):
                ex, rh = take(i, cx, cr)
                ei = row[i, 2]
                w = cw
                if i == l - 1:
                    w = R(-b[l])
                    rh = R(rh + row[l, 2])
                inv = one / R(R(ex - a[i]) + w)
                rr, cc, om, lam = rh * inv, a[i] * inv, w * inv, ex * inv
                row[i] = (rr, cc, om)
                Gs, Bs, Ds = R(Gs + rr * P), R(Bs + om * P), R(Ds + lam * P)
                P = R(P * -cc)
                if i > r:
                    cx, cr, cw = R(-b[i] * lam), R(ei - b[i] * rr), R(-b[i] * om)
                else:
                    jacc[ps[i]] += np.float64(-b[i] * lam), np.float64(ei - b[i] * rr)
                    sepv[lk, 1] = b[i] * om
            sepv[lk, 0], sepv[lk, 2], sepv[lk, 3] = a[l] * P, -a[l] * Ds, -a[l] * Gs
    seps = info["seps"]                                     # S2
    for k in range(len(seps) - 1, -1, -1):
        s, sp, seg = seps[k]
        ex, rh = take(s, R(0), R(0))
        A, B, eup = a[s], b[s], row[s, 2]
        if seg >= 0:
            A, B = sepv[k, 0], sepv[k, 1]
            ex = R(ex + sepv[k, 2])
            rh = R(rh + sepv[k, 3])
            eup = R(0)
        if k == 0:
            row[s, 0] = rh / ex
            break
        inv = one / R(ex - A)
        row[s, 0], row[s, 1] = rh * inv, A * inv
        jacc[js[seps[sp, 0]]] += np.float64(-B * (ex * inv)), np.float64(eup - B * row[s, 0])
    x = np.zeros(n, dtype=R)
    for k, (s, sp, seg) in enumerate(seps):
        x[s] = row[s, 0] if k == 0 else R(row[s, 0] - row[s, 1] * jx[js[seps[sp, 0]]])
        jx[js[s]] = x[s]
    for (r, u, l, lk, lo, hi) in info["comps"]:             # S3
        if l >= 0:
            xp, xl = jx[js[u]], jx[js[l]]
            for i in range(r, l):
                x[i] = R(row[i, 0] - row[i, 1] * xp + row[i, 2] * xl)
                xp = x[i]
                if js[i] >= 0:
                    jx[js[i]] = x[i]
        xprev = R(0)
        for i in range(lo, hi):
            xp = xprev if ps[i] < 0 else jx[ps[i]]
            x[i] = R(row[i, 0] - row[i, 1] * xp)
            if js[i] >= 0:
                jx[js[i]] = x[i]
            xprev = x[i]
    return x


def _exact_tree_solve(par, a, b, ex_own, rhs, e):
    """Exact rational solve of the tree system (Hines order, no rounding)."""
    from fractions import Fraction as F
    n = par.size
    d = [F(float(v)) for v in ex_own]
    r = [F(float(v)) for v in rhs]
    for i in range(1, n):
        d[i] -= F(float(a[i]))
        d[par[i]] -= F(float(b[i]))
        r[par[i]] += F(float(e[i]))
    for i in range(n - 1, 0, -1):
        f = F(float(b[i])) / d[i]
        d[par[i]] -= f * F(float(a[i]))
        r[par[i]] -= f * r[i]
    x = [F(0)] * n
    x[0] = r[0] / d[0]
    for i in range(1, n):
        x[i] = (r[i] - F(float(a[i])) * x[par[i]]) / d[i]
    return np.array([float(v) for v in x])


@pytest.mark.parametrize("name", list(CELLS))
@pytest.mark.parametrize("W", WARPS)
def test_split_solve_matches_dense(ngpu_built, name, W):
    cell = CELLS[name]
    info = Model(cell).split_info(W)
    par, a, b = _internal(cell, info)
    n = cell.n_nodes
    rng = np.random.default_rng(W * 1000 + n)
    ex = rng.uniform(0.01, 2.0, n) + 0.04
    rhs = rng.normal(0, 1, n)
    e = rng.normal(0, 0.1, n)
    e[0] = 0.0
    x = _emulate(par, a, b, info, ex, rhs, e)
    # dense: row i: d_i x_i + a_i x_p + sum_c b_c x_c = rhs_i + sum_c e_c,
    # d_i = ex_i - a_i - sum_c b_c
    d = ex - a
    d[0] = ex[0]
    np.add.at(d, par[1:], -b[1:])
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


def _shipped_ttpc512():
    from pathlib import Path
    from neurogpu_b200 import formats
    gold = Path(__file__).resolve().parent / "golden" / "ttpc512"
    return formats.read_data_dir(gold, stim_index=0, params_file="AllParams_reference.csv").cell


def _assembled_rows(par, a, b, cm, has_chan, rng, dt=0.1):
    """One step's rows as the FP32 kernel assembles them at a uniform
    voltage: excess g + cm/dt, right-hand sides from channel currents."""
    f = np.float32
    n = par.size
    dv = np.zeros(n, dtype=f)
    g = np.where(has_chan, rng.uniform(0.0, 0.05, n), 0.0).astype(f)
    ex = (g + (cm / (dt * 1000.0)).astype(f)).astype(f)
    I = np.where(has_chan, rng.normal(0, 0.5, n), 0.0).astype(f)
    rhs = (-I - a.astype(f) * dv).astype(f)
    e = (b.astype(f) * dv).astype(f)
    e[0] = 0
    return ex, rhs, e


def _unmerged_model(cell):
    """A model that keeps every node (stiff-edge merging off)."""
    import os
    old = os.environ.get("NGPU_CONTRACT")
    os.environ["NGPU_CONTRACT"] = "0"
    try:
        return Model(cell)
    finally:
        if old is None:
            del os.environ["NGPU_CONTRACT"]
        else:
            os.environ["NGPU_CONTRACT"] = old


@pytest.mark.parametrize("W", [1, 4, 8])
def test_fp32_excess_form_survives_extreme_couplings(ngpu_built, W):
    """The reference's shipped 512-node TTPC model joins a 12-node section of
    ~3e21 couplings to the rest of the cell through ~1e10 couplings (near
    zero-area compartments).  Eliminating with full diagonals in FP32 cancels
    the outer couplings away (errors of volts); the excess form keeps every
    update a sum of nonnegative terms and stays within FP32 rounding of the
    exact solution (the elimination alone; axial right-hand-side terms are
    zero at a uniform voltage)."""
    cell = _shipped_ttpc512()
    info = _unmerged_model(cell).split_info(W)
    par, a, b = _internal(cell, info)
    perm = info["perm"]
    cm = cell.cm[perm]
    has_chan = cell.mech_mask[:, perm].any(axis=0)
    rng = np.random.default_rng(W)
    ex, rhs, e = _assembled_rows(par, a, b, cm, has_chan, rng)
    exact = _exact_tree_solve(par, a.astype(np.float32), b.astype(np.float32), ex, rhs, e)
    got = _emulate(par, a, b, info, ex, rhs, e, dtype=np.float32).astype(np.float64)
    phys = has_chan | (cm > 0)
    err = np.abs(got - exact)[phys]
    scale = np.max(np.abs(exact[phys]))
    assert np.max(err) <= 1e-6 * scale
    # the conventional FP32 elimination on the same rows: diagonals cancel,
    # some to exactly zero
    f = np.float32
    with np.errstate(all="ignore"):
        d = (ex - a.astype(f)).astype(f)
        d[0] = ex[0]
        r = rhs.copy()
        for i in range(1, par.size):
            d[par[i]] = f(d[par[i]] - f(b[i]))
            r[par[i]] = f(r[par[i]] + e[i])
        for i in range(par.size - 1, 0, -1):
            q = f(f(b[i]) / d[i])
            d[par[i]] = f(d[par[i]] - q * f(a[i]))
            r[par[i]] = f(r[par[i]] - q * r[i])
        xc = np.zeros(par.size, dtype=f)
        xc[0] = r[0] / d[0]
        for i in range(1, par.size):
            xc[i] = (r[i] - f(a[i]) * xc[par[i]]) / d[i]
        errc = np.abs(xc.astype(np.float64) - exact)[phys]
    assert not np.all(np.isfinite(errc)) or np.max(errc) > 1e-2 * scale


def test_stiff_edge_merging(ngpu_built):
    """The shipped model's two stiff groups (nodes 2-14 and 112, 159-161,
    edge conductances 1e9..1e10 against a median of 1e-1.7) become one
    internal node each; the merged system's couplings are ordinary, and one
    step's exact solution at every node equals the unmerged system's to
    the stiffness ratio.  Synthetic cells keep every node."""
    cell = _shipped_ttpc512()
    M = Model(cell)
    nd, ar = M.nodes(), M.arrays()
    ni = nd["node_internal"]
    assert nd["n_internal"] == cell.n_nodes - 15
    assert len(set(ni[[2] + list(range(3, 15))])) == 1 and len(set(ni[[112, 159, 160, 161]])) == 1
    assert len(set(ni.tolist())) == nd["n_internal"]
    assert np.abs(ar["a"][1:]).max() < 1e3 and np.abs(ar["b"][1:]).max() < 1e3
    rng = np.random.default_rng(0)
    n = cell.n_nodes
    has_chan = cell.mech_mask.any(axis=0)
    g = np.where(has_chan, rng.uniform(0, 0.05, n), 0)
    ex = g + cell.cm / 100.0
    rhs = np.zeros(n)
    rhs[1] = 100 * 2.0 / 1437.06      # a 2 nA step into the soma
    x = _exact_tree_solve(cell.parent, cell.a, cell.b, ex, rhs, np.zeros(n))
    perm = M.split_info(1)["perm"]    # internal node -> representative caller node
    G = nd["n_internal"]
    rhs_g = np.zeros(G)
    rhs_g[ni[1]] = rhs[1] * nd["density_scale"][1]
    xg = _exact_tree_solve(ar["parent"], ar["a"], ar["b"], g[perm] + ar["cm"] / 100.0, rhs_g, np.zeros(G))
    assert np.max(np.abs(x - xg[ni])) <= 1e-8 * np.max(np.abs(x))
    for c in CELLS.values():
        assert Model(c).nodes()["n_internal"] == c.n_nodes


def test_shaped_simulation_rejects_bad_shapes(ngpu_built):
    """ngpu_sim_create_shaped checks its warp and item counts before any
    device work."""
    import ctypes as C

    from neurogpu_b200 import _ffi, configs
    from neurogpu_b200.sim import Model
    w = configs.passive_cable(n_sets=2, t_stop=1.0)
    m = Model(w.cell)
    L = _ffi.lib()
    h = C.c_void_p()
    assert L.ngpu_sim_create_shaped(m.handle, 2, 1, 0, 4, 9, C.byref(h)) == -1
    assert b"items_per_warp" in L.ngpu_last_error()
    assert L.ngpu_sim_create_shaped(m.handle, 2, 1, 0, 4, -1, C.byref(h)) == -1
    assert L.ngpu_sim_create_shaped(m.handle, 2, 1, 0, 9, 2, C.byref(h)) == -1
