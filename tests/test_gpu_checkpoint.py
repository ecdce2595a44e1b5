"""Checkpoint and resume of an ALI run through the C ABI.

A run stopped after ten iterations (two of them Ng steps) and written in
Magritte's text layout (populations and the three previous iterates), then
read into a new Simulation of the same model read back from its model
folder, continues exactly as the uninterrupted run: the populations after
ten more iterations are bit-identical in FP64.  The reference restarts its
Ng cadence on every call of compute_level_populations
(src/Simulation/sim_lines.tpp:86-118), as this library does, so the split
falls after an Ng step.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation, io_text

pytestmark = pytest.mark.gpu


def setup(model):
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    return sim


def test_checkpoint_resume_is_exact(gpu, tmp_path):
    model = M.wind_model(10, seed=7, nlev=5, nside=1, name="wind10")
    straight = setup(model)
    straight.compute_level_populations(True, 20, "fp64", tol_max_rel=1e-30)
    first = setup(model)
    first.compute_level_populations(True, 10, "fp64", tol_max_rel=1e-30)
    folder = str(tmp_path / "run") + "/"
    io_text.write_model(model, folder)
    first.write_checkpoint(folder)
    first.close()
    resumed = setup(io_text.read_model(folder))
    resumed.read_checkpoint(folder)
    resumed.compute_level_populations(True, 10, "fp64", tol_max_rel=1e-30)
    assert np.array_equal(resumed.population, straight.population)
    assert np.array_equal(np.array(resumed.error_max), np.array(straight.error_max[10:]))
