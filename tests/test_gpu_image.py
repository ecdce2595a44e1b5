"""Images through the C ABI against the CPU oracle (FP64, 1e-6 relative).

``mgr_compute_image`` traces both rays of every cell in the rest frame and
solves each ray pair for the intensities leaving through its two far ends,
as ``Simulation::compute_and_write_image`` does
(``src/Simulation/sim_radiation.tpp:348-478``); the oracle restates that
path and is itself checked bit-exact against the reference's compiled C++
(tests/test_reference_pin.py).  Cases: the static lattice, a wind (rest-
frame Doppler shifts up to many line widths) and a turbulent cloud with
Doppler sub-points, at LTE and at populations after three ALI iterations.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

import oracle

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6


def rel_err(a, b):
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    return float(np.nanmax(r))


CASES = [
    (M.config1, 0, 2e-4),
    (lambda: M.wind_model(10, seed=7, nlev=5, nside=1, name="wind10"), 1, 2e-5),
    (lambda: M.turbulent_cloud(6, seed=903, npairs=12, name="turb6"), 3, 3e-5),
]


@pytest.mark.parametrize("make,ray,width", CASES)
@pytest.mark.parametrize("iterate", [False, True])
def test_image_matches_oracle(gpu, make, ray, width, iterate):
    model = make()
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    if iterate:
        sim.compute_level_populations(True, 3, "fp64", tol_max_rel=1e-30)
    img = sim.compute_image(ray, width)
    orc = oracle.Oracle(model).setup()
    orc.set_populations(sim.population)
    orc.compute_spectral_discretisation_image(width)
    I_m, I_p = orc.compute_image(ray)
    assert np.array_equal(img["nu"], orc.nu[0])
    assert rel_err(img["I_m"], I_m) < FP64_RTOL
    assert rel_err(img["I_p"], I_p) < FP64_RTOL
    # Image::set_coordinates (Simulation/Image/image.cpp:86-127)
    r = model.rays[ray]
    den = np.sqrt(r[0] ** 2 + r[1] ** 2)
    x, y, z = model.position.T
    if den != 0.0:
        X = (r[1] / den) * x + (-r[0] / den) * y
        Y = (r[0] * r[2] / den) * x + (r[1] * r[2] / den) * y + (-den) * z
    else:
        X, Y = x, y
    scale = 1e-13 * np.abs(model.position).max()
    assert np.allclose(img["ImX"], X, rtol=0.0, atol=scale)
    assert np.allclose(img["ImY"], Y, rtol=0.0, atol=scale)
    # the radiation field's own grid is untouched by the image
    sim.compute_radiation_field("fp64", keep_J=True)
    orc2 = oracle.Oracle(model).setup()
    orc2.set_populations(sim.population)
    orc2.compute_radiation_field()
    assert rel_err(sim.J, orc2.J) < FP64_RTOL
