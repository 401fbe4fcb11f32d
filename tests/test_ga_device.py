"""Device genetic-algorithm steps (csrc/ga.cuh, ngpu_ga_*) against their
numpy restatement (oracle/ga_numpy.py).

CPU: the restatement's random stream against SplitMix64's published
sequence and against the header's own host-callable functions compiled
here; non-dominated sorting and crowding on hand-worked cases; operator
properties; argument checks of the C entry points (rejected before any GPU
call).  GPU: the kernels against the restatement on the same inputs --
children to 1e-12 (pow may differ in the last bit), survivor indices, front
ranks and crowding distances exactly -- over edge cases (one individual,
ties, duplicates, NaN scores, sizes that are not powers of two); then the
device-resident GA loop."""
import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import ga_numpy as G  # noqa: E402


def test_stream_is_splitmix64():
    # the first two outputs of SplitMix64 from state 0 (state advances by the golden gamma)
    assert int(G.splitmix64(0)) == 0xE220A8397B1DCDAF
    assert int(G.splitmix64(0x9E3779B97F4A7C15)) == 0x6E789E6AA1B965F4
    u = G.uniform(G.ga_key(7, 3), np.arange(20000, dtype=np.uint64), 5)
    assert 0.0 <= u.min() and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01
    k = G.index(G.ga_key(7, 3), np.arange(20000, dtype=np.uint64), 1, 13)
    assert k.min() == 0 and k.max() == 12 and np.all(np.abs(np.bincount(k) / 20000 - 1 / 13) < 0.01)


HOST_PROBE = r'''
#include <stdint.h>
#include "ga.cuh"
extern "C" uint64_t probe_key(uint64_t seed, uint64_t gen) { return ngpu::ga_key(seed, gen); }
extern "C" uint64_t probe_mix(uint64_t x) { return ngpu::splitmix64(x); }
extern "C" uint64_t probe_order(double x) { return ngpu::ga_order_key(x); }
'''


def test_header_stream_and_order_keys_match(tmp_path):
    """The kernels' host-callable stream and sort keys, compiled from
    csrc/ga.cuh, against the restatement."""
    (tmp_path / "p.cu").write_text(HOST_PROBE)
    r = subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "-Wno-deprecated-gpu-targets",
                        "-I", str(ROOT / "neurogpu_b200" / "csrc"), str(tmp_path / "p.cu"), "-o",
                        str(tmp_path / "libp.so")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    L = C.CDLL(str(tmp_path / "libp.so"))
    for fn in (L.probe_key, L.probe_mix, L.probe_order):
        fn.restype = C.c_uint64
    L.probe_key.argtypes = [C.c_uint64, C.c_uint64]
    L.probe_mix.argtypes = [C.c_uint64]
    L.probe_order.argtypes = [C.c_double]
    for seed, gen in ((0, 0), (1, 2), (2 ** 63 + 5, 77)):
        assert L.probe_key(seed, gen) == int(G.ga_key(seed, gen))
    for x in (0, 1, 12345, 2 ** 64 - 1):
        assert L.probe_mix(x) == int(G.splitmix64(x))
    xs = [-np.inf, -1e300, -1.0, -1e-300, -0.0, 0.0, 1e-300, 1.0, 1e300, np.inf, np.nan]
    keys = [L.probe_order(x) for x in xs]
    assert keys == sorted(keys) and keys[4] == keys[5] and len(set(keys)) == len(xs) - 1


def test_fronts_and_crowding_hand_worked():
    # two objectives: front 0 = (1,5) (2,3) (4,1); front 1 = (2,5) (3,4) (5,2); front 2 = (5,5)
    obj = np.array([[1, 5], [2, 3], [4, 1], [2, 5], [3, 4], [5, 2], [5, 5]], dtype=float)
    rank = G.fronts(obj)
    assert list(rank) == [0, 0, 0, 1, 1, 1, 2]
    crowd = G.crowding(obj, rank)
    # front 0 in objective 0: 1, 2, 4 (range 3) -> middle (4 - 1) / 3; objective 1: 1, 3, 5 -> (5 - 1) / 4
    assert np.isinf(crowd[0]) and np.isinf(crowd[2]) and crowd[1] == pytest.approx(1.0 + 1.0)
    assert np.isinf(crowd[6])
    idx, rk, cr, nf = G.select_nsga2(obj, 4)
    assert nf == 3 and list(idx[:3]) == [0, 2, 1] and rk[idx[3]] == 1
    # duplicates do not dominate each other; NaN counts as +inf
    dup = np.array([[1.0, 1.0], [1.0, 1.0], [np.nan, 0.5], [2.0, 2.0]])
    assert list(G.fronts(dup)) == [0, 0, 0, 1]


def test_offspring_properties():
    rng = np.random.default_rng(0)
    pop = rng.uniform(-1, 1, (50, 12))
    rank = np.zeros(50, dtype=np.int64)
    crowd = rng.normal(size=50)
    kids = G.offspring(pop, rank, crowd, 4000, -1.0, 1.0, 10.0, 20.0, 0.9, 1 / 12, 3, 1)
    assert kids.shape == (4000, 12) and kids.min() >= -1.0 and kids.max() <= 1.0
    # no crossover, no mutation: every child is a tournament winner, copied
    same = G.offspring(pop, rank, crowd, 500, -1.0, 1.0, 10.0, 20.0, 0.0, 0.0, 3, 1)
    rows = {tuple(r) for r in pop}
    assert all(tuple(r) in rows for r in same)
    # binary tournaments favour higher crowding: the copied parents' mean crowding is above the population's
    win = [int(np.nonzero(np.all(pop == r, axis=1))[0][0]) for r in same]
    assert crowd[win].mean() > crowd.mean() + 0.3


def test_entry_points_reject_bad_arguments(ngpu_built):
    from neurogpu_b200 import _ffi
    L = _ffi.lib()
    d = C.c_void_p(16)   # never dereferenced: the checks come first
    assert L.ngpu_ga_offspring(None, d, d, 4, 3, 8, -1.0, 1.0, 10.0, 20.0, 0.9, 0.3, 0, 0, d, None) == -1
    assert L.ngpu_ga_offspring(d, d, d, 0, 3, 8, -1.0, 1.0, 10.0, 20.0, 0.9, 0.3, 0, 0, d, None) == -1
    assert L.ngpu_ga_offspring(d, d, d, 4, 3, 8, 1.0, -1.0, 10.0, 20.0, 0.9, 0.3, 0, 0, d, None) == -1
    assert L.ngpu_ga_select_truncation(d, 10, 11, d, None) == -1
    assert L.ngpu_ga_select_nsga2(d, 40000, 2, 10, d, d, d, d, None) == -1
    assert L.ngpu_ga_select_nsga2(d, 100, 193, 10, d, d, d, d, None) == -1
    assert b"objectives" in L.ngpu_last_error()


# ------------------------------------------------------------------- GPU
def _cuda(x, dtype=None):
    import torch
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("mu,n_genes,n_kids,seed,gen", [(1, 1, 5, 0, 0), (300, 12, 1000, 42, 7),
                                                        (64, 40, 257, 2 ** 64 - 1, 123)])
def test_offspring_kernel_matches_restatement(ngpu_built, mu, n_genes, n_kids, seed, gen):
    import torch

    from neurogpu_b200.ga_device import DeviceGA
    rng = np.random.default_rng(mu + n_genes)
    pop = rng.uniform(-1, 1, (mu, n_genes))
    pop[: mu // 3, 0] = 1.0                         # genes on the bound
    if mu > 4:
        pop[1] = pop[0]                             # identical parents: no crossover spread
    rank = rng.integers(0, 3, mu).astype(np.int32)
    crowd = np.round(rng.uniform(0, 2, mu), 1)      # ties
    crowd[::7] = np.inf
    ga = DeviceGA(n_genes, eta_c=10.0, eta_m=20.0, cx_prob=0.9, p_mut=0.3, seed=seed)
    got = ga.offspring(_cuda(pop), _cuda(rank, torch.int32), _cuda(crowd), n_kids, gen).cpu().numpy()
    want = G.offspring(pop, rank, crowd, n_kids, -1.0, 1.0, 10.0, 20.0, 0.9, 0.3, seed, gen)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
    assert got.min() >= -1.0 and got.max() <= 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("n,mu", [(1, 1), (7, 3), (1000, 500), (5000, 5000), (20000, 4096)])
def test_truncation_matches_restatement(ngpu_built, n, mu):
    from neurogpu_b200.ga_device import select_truncation
    rng = np.random.default_rng(n)
    s = np.round(rng.normal(size=n), 2)             # many ties
    s[::11] = np.nan
    if n > 3:
        s[1], s[2] = -0.0, 0.0
    got = select_truncation(_cuda(s), mu).cpu().numpy()
    np.testing.assert_array_equal(got, G.select_truncation(s, mu))


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,mu", [(1, 1, 1), (2, 3, 1), (100, 2, 50), (333, 1, 100), (1000, 5, 600),
                                    (4096, 60, 2048)])
def test_nsga2_matches_restatement(ngpu_built, n, m, mu):
    from neurogpu_b200.ga_device import select_nsga2
    rng = np.random.default_rng(n * 7 + m)
    obj = np.round(rng.uniform(0, 3, (n, m)), 1)    # ties in every objective
    if n > 10:
        obj[5] = obj[4]                             # a duplicate
        obj[9, 0] = np.nan
    idx, rank, crowd, nf = select_nsga2(_cuda(obj), mu)
    w_idx, w_rank, w_crowd, w_nf = G.select_nsga2(obj, mu)
    np.testing.assert_array_equal(rank.cpu().numpy(), w_rank)
    np.testing.assert_array_equal(crowd.cpu().numpy(), w_crowd)
    np.testing.assert_array_equal(idx.cpu().numpy(), w_idx)
    assert int(nf) == w_nf


@pytest.mark.gpu
@pytest.mark.parametrize("selector", ["truncation", "nsga2"])
def test_device_ga_loop(ngpu_built, selector):
    """Two generations of the device-resident GA on a small fitting problem;
    its simulation path gives the host path's features."""
    import torch

    from neurogpu_b200 import ga
    prob = ga.FitProblem(n_comp=120, t_stop=120.0, stim_on=20.0, stim_off=100.0, levels=(0.5, 1.0))
    u = np.random.default_rng(1).uniform(-1, 1, (16, prob.n_params))
    f_host = prob.simulate(u)
    f_dev = prob.simulate_device(_cuda(u)).cpu().numpy()
    np.testing.assert_array_equal(f_dev[..., 0], f_host[..., 0])        # spike counts
    np.testing.assert_allclose(f_dev, f_host, rtol=1e-4, atol=1e-3)
    n0 = prob.sim_count
    res = ga.run_device(prob, pop_size=64, generations=2, seed=3, selector=selector)
    assert len(res.best) == 2 and prob.sim_count - n0 == 64 * 3
    assert res.best_u.shape == (prob.n_params,) and np.all(np.abs(res.best_u) <= 1.0)
    if selector == "truncation":
        assert res.best[1] <= res.best[0]
    torch.cuda.synchronize()
