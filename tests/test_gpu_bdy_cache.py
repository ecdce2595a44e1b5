"""The staged mixed solve reads the far ends' boundary intensities from a
cache filled once per trace store.  These tests check that the cache follows
the state it depends on: the traces (a new model, an origin range, traces
rebuilt per batch of origins) and agrees with the oracle."""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

import oracle

pytestmark = pytest.mark.gpu

MIXED_RTOL = 1e-4


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    return float(np.nanmax(r))


def ready(sim):
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    return sim


def mixed_solve(sim):
    sim.compute_radiation_field("mixed", keep_J=True)
    assert sim.tuning("mixed")["kernel"] == "staged"
    return sim.J.copy(), sim.Jlin.copy(), sim.Lambda.copy()


def test_new_model_on_same_handle(gpu):
    """A second model uploaded to a handle that solved another: the same
    results as a fresh handle (bit for bit), and the oracle's to 1e-4."""
    a = M.wind_model(10, seed=7, nlev=5, nside=1, name="wind10")
    b = M.wind_model(11, seed=3, nlev=5, nside=1, vmax=40e3, name="wind11")
    sim = ready(Simulation(a))
    mixed_solve(sim)
    sim.read(b)
    ready(sim)
    J1, Jl1, L1 = mixed_solve(sim)
    fresh = ready(Simulation(b))
    J2, Jl2, L2 = mixed_solve(fresh)
    assert np.array_equal(J1, J2) and np.array_equal(Jl1, Jl2) and np.array_equal(L1, L2)
    orc = oracle.Oracle(b).setup()
    orc.compute_radiation_field()
    orc.compute_Jeff()
    assert rel_err(J1, orc.J) < MIXED_RTOL
    assert rel_err(L1, orc.Ls) < MIXED_RTOL


def test_origin_range_and_batches(gpu):
    """An origin range, and traces rebuilt per batch of origins: each origin's
    J, Jlin and ALO equal the whole stored solve's bit for bit."""
    model = M.wind_model(10, seed=5, nlev=5, nside=1, name="wind10")
    sim = ready(Simulation(model))
    J0, Jl0, L0 = mixed_solve(sim)
    b, e = 320, 640
    sim.set_origin_range(b, e)
    _, Jl1, L1 = mixed_solve(sim)
    assert np.array_equal(Jl1[b:e], Jl0[b:e]) and np.array_equal(L1[b:e], L0[b:e])
    sim.set_origin_range(0, model.ncells)
    sim.set_trace_budget(1 << 19)
    J2, Jl2, L2 = mixed_solve(sim)
    assert np.array_equal(J2, J0) and np.array_equal(Jl2, Jl0) and np.array_equal(L2, L0)
