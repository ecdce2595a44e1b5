"""Batches of independent models, graph-replayed iterations and the
autotuner, through the C ABI.

A batch (``concat_models`` + ``mgr_set_segments``) must give every member
what a Simulation of that member alone gives: in FP64 the same populations
(the per-model Ng and convergence reductions run in a fixed order, so the
arithmetic is the solo run's) and the same iteration count; in mixed
precision agreement to 1e-4.  Graph replay and every autotuner candidate
must reproduce the plain launches bit for bit.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

pytestmark = pytest.mark.gpu

TOL = 1e-6


def members():
    """Three small winds of uneven size sharing species and rays."""
    out = []
    for i, (n, rho0, T0, vmax) in enumerate([(6, 1e13, 300.0, 8e3), (9, 3e14, 1500.0, 25e3),
                                              (7, 1e15, 800.0, 15e3)]):
        out.append(M.wind_model(n, seed=40 + i, nlev=6, npairs=6, rho0=rho0, T0=T0, vmax=vmax,
                                name=f"member{i}", species_seed=40, ray_seed=40))
    return out


def solve(model, precision="fp64", use_graph=False, tol=TOL):
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    it = sim.compute_level_populations(True, 200, precision, tol_max_rel=tol,
                                       use_graph=use_graph)
    return sim, it


def test_batch_matches_solo_fp64(gpu):
    ms = members()
    solo = [solve(m) for m in ms]
    batch = M.concat_models(ms)
    sim, it = solve(batch)
    assert sim.converged
    _, iters = sim.segment_results()
    pop = sim.population
    seg = batch.meta["segments"]
    for s, (ssim, sit) in enumerate(solo):
        assert iters[s] == sit
        ref = ssim.population
        got = pop[seg[s]:seg[s + 1]]
        assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-12
    assert it == max(sit for _, sit in solo)


def test_batch_matches_solo_mixed(gpu):
    ms = members()
    batch = M.concat_models(ms)
    sim, _ = solve(batch, "mixed")
    assert sim.converged
    seg = batch.meta["segments"]
    for s, m in enumerate(ms):
        ref, _ = solve(m, "fp64")
        got = sim.population[seg[s]:seg[s + 1]]
        rel = np.abs(got - ref.population) / np.maximum(ref.population, 1e-300)
        assert rel[ref.population > 1e-10 * m.population_tot[:, None]].max() < 1e-4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_is_exact(gpu, precision):
    for model in (M.wind_model(8, seed=3, nlev=5, nside=1), M.concat_models(members())):
        a, ia = solve(model, precision, use_graph=False)
        b, ib = solve(model, precision, use_graph=True)
        assert ia == ib
        assert np.array_equal(a.population, b.population)
        assert a.error_max == b.error_max


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotuner_candidates_agree(gpu, precision):
    model = M.wind_model(10, seed=5, nlev=5, nside=1)
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    sim.set_autotune(2)
    outs = []
    for _ in range(4):
        sim.compute_radiation_field(precision, keep_J=True)
        outs.append((sim.J.copy(), sim.Jlin.copy(), sim.Lambda.copy()))
    t = sim.tuning(precision)
    assert t["tuned"] and all(x > 0 for x in t["ms"])
    assert t["min_blocks"] in (6, 7, 8)
    assert t["kernel"] == "staged"
    for o in outs[1:]:
        for x, y in zip(o, outs[0]):
            assert np.array_equal(x, y)
