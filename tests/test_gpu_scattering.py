"""The formal solve with scattering terms through the C ABI, against the
CPU oracle (FP64, 1e-6 relative).

``mgr_compute_radiation_field_scattering`` restates the reference's
``Simulation::setup_using_scattering`` and ``RayPair::solve_using_scattering``
(``src/Simulation/simulation.tpp:51-171``,
``src/Simulation/Raypair/raypair_solver.tpp:10-190``) for every ray pair and
origin; the oracle's restatement of the same functions is checked against
the reference's compiled C++ in tests/test_reference_pin.py.  The test sets
scattering terms U, V of emissivity size (the reference adds U to the
emissivity), compares u and v at the origins, J, Jlin and the ALO, then
forms the next terms with ``mgr_calc_U_and_V`` (``Radiation::calc_U_and_V``,
which sums intensities over the pairs) and checks those against the
oracle's.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

import oracle

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6


def rel_err(a, b, floor=0.0):
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.maximum(np.abs(b), floor)
    r[a == b] = 0.0
    return float(np.nanmax(r))


KB, AMU, CC = 1.38064852e-23, 1.66053904e-27, 2.99792458e8


def emissivity_on_grid(model, orc):
    """The line emissivity at every cell's own bins, as get_eta_and_chi
    sums it: eps_l nu phi_l(nu) over the lines within 11 widths."""
    pw = np.sqrt(2.0 * KB / (AMU * CC ** 2) * model.linedata.inverse_mass * model.temperature
                 + model.vturb2)
    nu = orc.nu                                    # [N, nf]
    line = model.linedata.frequency                # [K]
    width = line[None, :] * pw[:, None]            # [N, K]
    diff = nu[:, :, None] - line[None, None, :]    # [N, nf, K]
    x = diff / width[:, None, :]
    phi = np.where(np.abs(x) <= 11.0, np.exp(-x * x) / (np.sqrt(np.pi) * width[:, None, :]), 0.0)
    return (orc.emissivity[:, None, :] * nu[:, :, None] * phi).sum(-1)


def terms(model, orc):
    """Scattering terms of emissivity size (the reference adds U to eta):
    fractions of the line emissivity varying with pair, cell and bin."""
    eta = emissivity_on_grid(model, orc)
    np_, N, nf = model.nrays // 2, model.ncells, model.nfreqs
    r = np.arange(np_)[:, None, None]
    p = np.arange(N)[None, :, None]
    f = np.arange(nf)[None, None, :]
    U = eta[None] * (0.3 + 0.05 * r) * (1.0 + 0.2 * np.sin(0.37 * p + 0.11 * f))
    V = eta[None] * 0.1 * np.cos(0.23 * p + 0.07 * f + 0.5 * r)
    # zero beyond 3 Doppler widths of each line: rescale_U_and_V holds the
    # edge value beyond a cell's grid, where the opacity that U is divided
    # by falls to its 1e-26 floor
    outer = np.tile(np.abs(model.quad_roots) >= 3.0, model.nlines)
    U[:, :, outer] = 0.0
    V[:, :, outer] = 0.0
    return U, V


@pytest.mark.parametrize("make", [
    M.config1,
    lambda: M.wind_model(10, seed=7, nlev=5, nside=1, name="wind10"),
    lambda: M.turbulent_cloud(6, seed=903, npairs=12, name="turb6"),
])
def test_scattering_solve_matches_oracle(gpu, make):
    model = make()
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    orc = oracle.Oracle(model).setup()
    U, V = terms(model, orc)
    sim.set_scattering_terms(U, V)
    sim.compute_radiation_field_scattering(keep_J=True)
    u, v = sim.scattering_uv()
    u_o, v_o = orc.compute_radiation_field_scattering(U, V)
    orc.compute_Jeff()
    # u and v change sign (the scattering terms enter through differences):
    # relative error with a floor of 1e-9 of u's largest value; v, a flux
    # that is a difference of the two directions' intensities (near zero in
    # the static lattice), relative to 1e-6 of its largest value, i.e. its
    # small values to 1e-12 of the flux scale
    assert rel_err(u, u_o, floor=1e-9 * np.abs(u_o).max()) < FP64_RTOL
    assert rel_err(v, v_o, floor=1e-6 * np.abs(v_o).max()) < FP64_RTOL
    # the scattering terms can drive J of the weakest lines slightly
    # negative: the same floor of 1e-9 of the largest value
    assert rel_err(sim.J, orc.J, floor=1e-9 * np.abs(orc.J).max()) < FP64_RTOL
    assert rel_err(sim.Jlin, orc.Jlin, floor=1e-9 * np.abs(orc.Jlin).max()) < FP64_RTOL
    assert rel_err(sim.Lambda, orc.Ls, floor=1e-9 * np.abs(orc.Ls).max()) < FP64_RTOL
    # the next scattering terms from this solve
    sim.calc_U_and_V()
    U2, V2 = sim.scattering_terms()
    U2_o, V2_o = orc.calc_U_and_V(u_o, v_o)
    # sums of u (and of v) over the pairs: the floors of u and v
    assert rel_err(U2, U2_o, floor=1e-9 * np.abs(U2_o).max()) < FP64_RTOL
    assert rel_err(V2, V2_o, floor=1e-6 * np.abs(V2_o).max()) < FP64_RTOL
