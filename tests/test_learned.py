"""Learned warm start: device forward/gradients against the numpy oracle
(oracle/mlp.py), and the gain of a trained network over the LTE start."""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation
from magritte_b200.learned import WarmStartNet, converged_samples, wind_family

from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def _random_batch(n, nlev, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 10)).astype(np.float32) * 3 + 5
    logits = rng.normal(size=(n, nlev))
    lte = (logits - np.log(np.exp(logits).sum(1, keepdims=True))).astype(np.float32)
    t = lte + rng.normal(scale=0.5, size=lte.shape)
    t = (t - np.log(np.exp(t).sum(1, keepdims=True))).astype(np.float32)
    t[:, -1] = np.log(1e-12)   # a level below the weight threshold
    return X, lte, t


def _random_net(nlev, seed):
    net = WarmStartNet(nlev).init(seed)
    rng = np.random.default_rng(seed + 1)
    net.params = (net.params + rng.normal(scale=0.05, size=net.params.shape)).astype(np.float32)
    net.feat_mean = rng.normal(size=10).astype(np.float32) + 5
    net.feat_istd = rng.uniform(0.2, 0.5, size=10).astype(np.float32)
    return net


@pytest.mark.parametrize("nlev", [2, 10, 21])
def test_forward_matches_numpy(gpu, nlev):
    X, _, _ = _random_batch(100, nlev, 1)
    net = _random_net(nlev, 2)
    got = net.forward(X)
    ref, _ = omlp.forward(net.params, net.feat_mean.astype(np.float64),
                          net.feat_istd.astype(np.float64), X, nlev)
    assert np.max(np.abs(got - ref)) < 1e-4 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("nlev", [2, 10, 21])
def test_gradients_match_numpy(gpu, nlev):
    X, lte, t = _random_batch(77, nlev, 3)
    net = _random_net(nlev, 4)
    loss, g = net.loss_grad(X, lte, t)
    loss_ref, g_ref = omlp.loss_and_grad(net.params, net.feat_mean.astype(np.float64),
                                         net.feat_istd.astype(np.float64), X, lte, t)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    scale = np.abs(g_ref).max()
    assert np.max(np.abs(g - g_ref)) <= 2e-4 * scale


def test_untrained_network_is_lte(gpu):
    model = M.wind_model(8, seed=3, nlev=6, nside=1)
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    lte = sim.population
    sim.warm_start(WarmStartNet(6).init(0))
    assert np.allclose(sim.population, lte, rtol=1e-5, atol=1e-12 * lte.max())


def test_trained_network_saves_iterations(gpu):
    """Train on eight small winds, then solve two held-out winds from the LTE
    start and from the learned start to the same tolerance: the learned start
    is at least twice as close to the converged populations (smaller first
    change) and never needs more iterations."""
    Xs, Ls, Ts = [], [], []
    for m in wind_family(12, 8, 500, nlev=6, nside=1):
        X, L, T, _ = converged_samples(m, precision="fp64", tol=1e-6, max_iter=400)
        Xs.append(X); Ls.append(L); Ts.append(T)
    net = WarmStartNet(6).init(0)
    hist = net.train(np.concatenate(Xs), np.concatenate(Ls), np.concatenate(Ts), epochs=150,
                     batch=1024, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0]
    for held in wind_family(12, 2, 900, nlev=6, nside=1):
        res = {}
        for start in ("lte", "learned"):
            sim = Simulation(held)
            sim.compute_spectral_discretisation()
            sim.compute_boundary_intensities()
            sim.compute_LTE_level_populations()
            if start == "learned":
                sim.warm_start(net)
            it = sim.compute_level_populations(True, 400, "fp64", tol_max_rel=1e-4)
            assert sim.converged
            res[start] = (it, sim.error_max[0])
            sim.close()
        print(held.name, "iterations, first change:", res)
        assert res["learned"][0] <= res["lte"][0]
        assert res["learned"][1] < 0.5 * res["lte"][1]
