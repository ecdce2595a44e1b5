"""The non-local ALO (mgr_set_n_off_diag) through the C ABI, against the CPU
oracle's restatement (FP64).

* The off-diagonal elements of every (cell, line, ray pair, side, distance)
  and their cells after one formal solve: 1e-6 relative (floor 1e-9 of the
  largest element), cells exact; J, Jlin and the diagonal ALO unchanged.
* Jeff with the non-local sums and one statistical-equilibrium solve of all
  cells as one system (block Jacobi on the device, the same on the oracle):
  populations 1e-6 on levels above 1e-6 of the cell's total, 1e-4 on the
  weaker levels down to 1e-10 (the per-cell LU rounding, as for the local
  ALO).
* The ALI iteration with n_off_diag = 2 to convergence: the same iteration
  count as the oracle, its populations, and the local ALO's fixed point.
* Batches and origin ranges refuse a non-local ALO with a status code.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation
from magritte_b200._capi import MagritteError

import oracle

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6


def rel(a, b, floor=0.0):
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.maximum(np.abs(b), floor)
    r[a == b] = 0.0
    return float(np.nanmax(r)) if r.size else 0.0


def check_pops(pop, ref, model, rtol):
    frac = ref / model.population_tot[:, None]
    big = frac > 1e-6
    weak = (frac > 1e-10) & ~big
    assert rel(pop[big], ref[big]) < rtol
    if weak.any():
        assert rel(pop[weak], ref[weak]) < max(rtol, 1e-4)


MODELS = [
    lambda: M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8"),
    lambda: M.turbulent_cloud(5, seed=903, npairs=12, name="turb5"),
]


def setup_pair(model, noff):
    sim = Simulation(model)
    sim.set_n_off_diag(noff)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    orc = oracle.Oracle(model).setup().set_n_off_diag(noff)
    return sim, orc


@pytest.mark.parametrize("make", MODELS)
@pytest.mark.parametrize("noff", [2, 3])
def test_offdiagonal_elements_match_oracle(gpu, make, noff):
    model = make()
    sim, orc = setup_pair(model, noff)
    sim.compute_radiation_field("fp64")
    orc.compute_radiation_field()
    Loff, nr = sim.alo_nonlocal()
    assert (nr == orc.Loff_nr).all()
    assert rel(Loff, orc.Loff, floor=1e-9 * np.abs(orc.Loff).max()) < FP64_RTOL
    assert rel(sim.Lambda, orc.Ls) < FP64_RTOL
    # Jeff with the non-local sums, then one solve of all cells' rate equations
    sim.compute_Jeff()
    orc.compute_Jeff()
    assert rel(sim.Jlin, orc.Jlin) < FP64_RTOL
    assert rel(sim.Jeff, orc.Jeff, floor=1e-9 * np.abs(orc.Jeff).max()) < FP64_RTOL
    sim.compute_level_populations_from_stateq()
    orc.compute_level_populations_from_stateq()
    assert orc.lu_errors == 0 and sim.nonlocal_sweeps() >= 1
    check_pops(sim.population, orc.pop, model, FP64_RTOL)


@pytest.mark.parametrize("make", MODELS)
def test_nonlocal_ali_matches_oracle_and_the_local_fixed_point(gpu, make):
    model = make()
    sim, orc = setup_pair(model, 2)
    it = sim.compute_level_populations(True, 60, "fp64", tol_max_rel=1e-6)
    it_o, hist_o = orc.compute_level_populations(True, 60, 1e-6)
    assert sim.converged and it == it_o
    check_pops(sim.population, orc.pop, model, FP64_RTOL)
    loc = Simulation(model)
    loc.compute_spectral_discretisation()
    loc.compute_boundary_intensities()
    loc.compute_LTE_level_populations()
    loc.compute_level_populations(True, 60, "fp64", tol_max_rel=1e-9)
    sel = loc.population > 1e-6 * model.population_tot[:, None]
    assert rel(sim.population[sel], loc.population[sel]) < 1e-5


def test_nonlocal_alo_needs_one_whole_model(gpu):
    members = [M.config4_member(i) for i in range(2)]
    batch = M.concat_models(members)
    sim = Simulation(batch)
    with pytest.raises(MagritteError):
        sim.set_n_off_diag(2)
    sim.set_n_off_diag(1)          # the diagonal ALO stays available
    single = Simulation(members[0])
    single.set_n_off_diag(2)
    with pytest.raises(MagritteError):
        single.set_origin_range(0, 32)
    with pytest.raises(MagritteError):
        single.set_n_off_diag(9)
