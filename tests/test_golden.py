"""The oracle still reproduces the committed golden fixtures (CPU), and the
device path matches them (GPU).  Fixtures: tests/golden/make_golden.py."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

CASES = sorted(make_golden.CASES)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))


def rel(a, b, floor=0.0):
    den = np.maximum(np.abs(b), floor)
    return float(np.max(np.abs(a - b) / den))


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(name):
    gold = load(name)
    out = make_golden.compute(name)
    for key in ("J", "Jlin", "Ls", "pop_lte"):
        assert np.array_equal(out[key], gold[key]), key
    floor = 1e-10 * np.abs(gold["pop_it3"]).max()
    assert rel(out["pop_it3"], gold["pop_it3"], floor) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_matches_golden(gpu, name):
    from magritte_b200 import Simulation
    gold = load(name)
    model = make_golden.CASES[name]()
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    assert rel(sim.population, gold["pop_lte"]) < 1e-12
    sim.compute_radiation_field("fp64", keep_J=True)
    assert rel(sim.J, gold["J"]) < 1e-6
    assert rel(sim.Jlin, gold["Jlin"]) < 1e-6
    assert rel(sim.Lambda, gold["Ls"]) < 1e-6
    sim.population = gold["pop_lte"]
    it = sim.compute_level_populations(True, 3, "fp64", tol_max_rel=1e-30)
    assert it == 3
    floor = 1e-10 * np.abs(gold["pop_it3"]).max()
    assert rel(sim.population, gold["pop_it3"], floor) < 1e-6
