"""The surrogate network (tcgen05 GEMMs, forward and backward) and the GA.

* gradients of every weight and bias against an FP64 numpy implementation
  of the same network on the same bf16 weights and inputs (the GPU path
  rounds activations to bf16 between layers: bound 3e-2 relative, cosine
  >= 0.999);
* training reduces the loss on a smooth map;
* what the trained network gains: on a small fitting problem, the 10 % of
  offspring it picks have much better true scores than a random 10 %;
* GA operators stay in bounds and SBX keeps the parents' mean on average
  (CPU)."""
import numpy as np
import pytest

from neurogpu_b200 import ga


def test_ga_operators_bounds_and_sbx_mean():
    rng = np.random.default_rng(0)
    a, b = rng.uniform(-1, 1, (4000, 12)), rng.uniform(-1, 1, (4000, 12))
    c1, c2 = ga.sbx(rng, a, b)
    assert np.all(np.abs(c1) <= 1) and np.all(np.abs(c2) <= 1)
    # bounded SBX spreads each child by its own bound distance: the pair's
    # mean matches the parents' on average, not per pair
    assert abs(np.mean((c1 + c2) / 2 - (a + b) / 2)) < 0.01
    m = ga.poly_mutate(rng, a)
    assert np.all(np.abs(m) <= 1) and 0 < np.mean(m != a) < 0.2
    score = rng.random(100)
    w = ga.tournament(rng, score, 10000)
    assert score[w].mean() < score.mean()
    x = ga._inputs(np.zeros((2, 12)), 3)
    assert x.shape == (6, 15) and np.array_equal(x[:, 12:], np.tile(np.eye(3), (2, 1)))


def _gelu(z):
    return 0.5 * z * (1 + np.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3)))


def _gelu_grad(z):
    t = np.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * 0.7978845608028654 * (1 + 3 * 0.044715 * z * z)


@pytest.mark.gpu
def test_gradients_match_fp64(ngpu_built):
    import torch
    from neurogpu_b200.surrogate import SurrogateMLP
    rng = np.random.default_rng(1)
    M, n_in, n_out = 300, 15, 20
    X = rng.normal(size=(M, n_in)).astype(np.float32)
    Y = rng.normal(size=(M, n_out)).astype(np.float32)
    net = SurrogateMLP(n_in, n_out, seed=3)
    loss, gW, gb = net.loss_and_grads(X, Y)
    # FP64 reference on the same bf16 weights / inputs
    Ws = [w.float().cpu().numpy().astype(np.float64) for w in net.Wb]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.b]
    x = torch.as_tensor(X).to(torch.bfloat16).float().numpy().astype(np.float64)
    h = np.zeros((M, net.k_in))
    h[:, :n_in] = x
    Hs, Zs = [h], []
    for k in range(3):
        z = Hs[-1] @ Ws[k].T + bs[k]
        Zs.append(z)
        Hs.append(_gelu(z))
    y = Hs[-1] @ Ws[3].T + bs[3]
    diff = y[:, :n_out] - Y
    assert float(loss) == pytest.approx(np.mean(diff ** 2), rel=2e-2)
    dy = np.zeros_like(y)
    dy[:, :n_out] = 2 * diff / (M * n_out)
    refW, refb = [None] * 4, [None] * 4
    refW[3], refb[3] = dy.T @ Hs[3], dy.sum(0)
    dh = dy @ Ws[3]
    for k in (2, 1, 0):
        dz = dh * _gelu_grad(Zs[k])
        refW[k], refb[k] = dz.T @ Hs[k], dz.sum(0)
        dh = dz @ Ws[k]
    for k in range(4):
        for got, ref in ((gW[k].cpu().numpy(), refW[k]), (gb[k].cpu().numpy(), refb[k])):
            rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            cos = float(np.sum(got * ref) / (np.linalg.norm(got) * np.linalg.norm(ref) + 1e-30))
            assert rel <= 3e-2 and cos >= 0.999, (k, rel, cos)


@pytest.mark.gpu
def test_training_reduces_loss(ngpu_built):
    from neurogpu_b200.surrogate import SurrogateMLP
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (8192, 15)).astype(np.float32)
    A = rng.normal(size=(15, 20))
    Y = (np.sin(X @ A) + 0.5 * (X @ A) ** 2).astype(np.float32)
    net = SurrogateMLP(15, 20, seed=0)
    hist = net.train(X, Y, epochs=40, batch=1024, lr=1e-3)
    assert hist[-1] < 0.1 * hist[0]


@pytest.mark.gpu
def test_surrogate_screening_beats_random_choice(ngpu_built):
    """What the network gains: offspring it ranks in the top 10 % score far
    better (true simulation) than a random 10 % of the same offspring."""
    from neurogpu_b200.surrogate import SurrogateMLP
    prob = ga.FitProblem(n_comp=200, t_stop=120.0, stim_on=20.0, stim_off=100.0, levels=(0.3, 0.8), rec_every=4,
                         seed=9)
    rng = np.random.default_rng(0)
    U = rng.uniform(-1, 1, (4096, prob.n_params))
    F = prob.simulate(U)
    net = SurrogateMLP(prob.n_params + prob.n_stim, F.shape[-1], seed=0)
    net.train(ga._inputs(U, prob.n_stim), F.reshape(-1, F.shape[-1]).astype(np.float32), epochs=40, batch=1024)
    cand = rng.uniform(-1, 1, (2000, prob.n_params))
    pred = net.predict(ga._inputs(cand, prob.n_stim)).cpu().numpy().reshape(2000, prob.n_stim, -1)
    top = np.argsort(prob.score(pred))[:200]
    true = prob.score(prob.simulate(cand))
    rand = rng.choice(2000, 200, replace=False)
    print(f"mean true score: surrogate top 10 % {true[top].mean():.3f}, random 10 % {true[rand].mean():.3f}, "
          f"best possible {np.sort(true)[:200].mean():.3f}")
    assert true[top].mean() < 0.5 * true[rand].mean()


@pytest.mark.gpu
def test_inputs_device_matches_host():
    import torch
    u = np.random.default_rng(1).uniform(-1, 1, (5, 12))
    got = ga.inputs_device(torch.tensor(u, device="cuda"), 3).cpu().numpy()
    np.testing.assert_array_equal(got, ga._inputs(u, 3))


@pytest.mark.gpu
def test_device_screened_ga_with_a_pretrained_surrogate(ngpu_built):
    """The surrogate trained once over the whole search space (independent of
    the target), then the screened GA with every step on the device: the
    best score never rises, each generation simulates the network's top 10 %
    (or, on a fallback, every offspring), and the error it measured is
    recorded per generation."""
    prob = ga.FitProblem(n_comp=120, t_stop=120.0, stim_on=20.0, stim_off=100.0, levels=(0.3, 0.8), rec_every=4,
                         seed=9)
    fit = ga.train_surrogate(prob, n_train=4096, epochs=8, seed=0)
    assert fit.n_train == 4096 and np.isfinite(fit.final_loss) and fit.sim_seconds > 0
    prob.sim_count = 0
    pop, gens = 256, 4
    res = ga.run_screened_device(prob, fit.net, pop, gens, seed=2)
    assert len(res.best) == gens and np.all(np.diff(res.best) <= 0)
    keep = int(round(0.1 * pop))
    expect = pop + sum(keep if m == "screened" else pop for _, _, m in res.notes)
    assert prob.sim_count == expect
    assert all(np.isfinite(e) for _, e, _ in res.notes)
    assert res.best_u.shape == (12,) and np.all(np.abs(res.best_u) <= 1)
