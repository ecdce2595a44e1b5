"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: traced points are bit-exact; J, Jlin, the ALO and level
populations agree to 1e-6 relative in FP64 mode (the measured gap is
~1e-12: the device elimination is algebraically the reference's but rounds
differently) and to 1e-4 in mixed mode.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

import oracle

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6
MIXED_RTOL = 1e-4


def rel_err(a, b, floor=0.0):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), floor)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / den
    r[(a == b)] = 0.0
    return float(np.nanmax(r)) if r.size else 0.0


def small_wind(n=10, nlev=5, seed=7):
    return M.wind_model(n, seed=seed, nlev=nlev, nside=1, name=f"wind{n}")


def broken_lattice():
    """6^3 lattice whose interior cell (2,2,2) has an empty neighbour list:
    every ray that enters it finds no neighbour ahead."""
    model = M.lattice_cloud(6, name="broken")
    p = 2 + 6 * (2 + 6 * 2)
    offs = model.nbr_offsets.copy()
    a, b = int(offs[p]), int(offs[p + 1])
    model.nbr_list = np.concatenate([model.nbr_list[:a], model.nbr_list[b:]])
    offs[p + 1:] -= (b - a)
    model.nbr_offsets = offs
    return model


def setup_pair(model, keep_J=True):
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    orc = oracle.Oracle(model).setup()
    if keep_J:
        sim.compute_radiation_field("fp64", keep_J=True)
    return sim, orc


@pytest.mark.parametrize("make", [M.config1, lambda: small_wind(10, 5, 7),
                                  lambda: M.wind_model(9, seed=3, nlev=4, nside=2, vmax=40e3),
                                  lambda: M.slab_1d(300, vmax=980.0)])
def test_traces_bit_exact(gpu, make):
    """Traced cells, shifts and increments equal the oracle's bit for bit.
    The 300-cell slab has walks longer than the counting pass's hop log
    holds (128 hops), which the fill searches again, beside shorter ones
    that it replays."""
    model = make()
    sim = Simulation(model)
    orc = oracle.Oracle(model)
    sim.trace()
    rng = np.random.default_rng(0)
    origins = rng.choice(model.ncells, size=min(model.ncells, 120), replace=False)
    for o in origins:
        for r in range(model.nrays):
            c1, s1, z1 = sim.trace_ray(int(o), r)
            c2, s2, z2 = orc.trace_ray(int(o), r)
            assert np.array_equal(c1, c2), (o, r)
            assert np.array_equal(s1, s2), (o, r)
            assert np.array_equal(z1, z2), (o, r)


def test_npoints_on_rays(gpu):
    model = small_wind(8, 4, 11)
    sim = Simulation(model)
    orc = oracle.Oracle(model)
    assert np.array_equal(sim.get_npoints_on_rays(), orc.get_npoints_on_rays())


@pytest.mark.parametrize("make", [M.config1, lambda: small_wind(10, 5, 7), M.config3,
                                  lambda: M.slab_1d(100, x_abund=1e-4, vmax=980.0)])
def test_radiation_field_fp64(gpu, make):
    model = make()
    sim, orc = setup_pair(model)
    orc.compute_radiation_field()
    assert orc.trace_errors == 0
    J = sim.J
    assert rel_err(J, orc.J) < FP64_RTOL
    orc.compute_Jeff()
    assert rel_err(sim.Jlin, orc.Jlin) < FP64_RTOL
    assert rel_err(sim.Lambda, orc.Ls) < FP64_RTOL
    sim.compute_Jeff()
    assert rel_err(sim.Jeff, orc.Jeff, floor=1e-3 * np.abs(orc.Jlin).max()) < FP64_RTOL


def test_radiation_field_subset_config2_shape(gpu):
    """The 64^3 wind at full size: J line integrals and ALO at a sample of
    origins against the oracle (which solves only those origins)."""
    model = M.config2()
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    sim.compute_radiation_field("fp64")
    orc = oracle.Oracle(model).setup()
    rng = np.random.default_rng(1)
    origins = np.sort(rng.choice(model.ncells, size=24, replace=False))
    orc.compute_radiation_field(origins=origins)
    orc.compute_Jeff()
    assert rel_err(sim.Jlin[origins], orc.Jlin[origins]) < FP64_RTOL
    assert rel_err(sim.Lambda[origins], orc.Ls[origins]) < FP64_RTOL


@pytest.mark.parametrize("ng_every", [0, 3])
def test_stateq_and_ng_iterations(gpu, ng_every):
    """Eight ALI iterations against the oracle: Ng at the 5th (the
    reference's cadence) or at the 4th and 8th (ng_every = 3)."""
    model = small_wind(10, 5, 7)
    sim, orc = setup_pair(model, keep_J=False)
    it_gpu = sim.compute_level_populations(use_Ng=True, max_niterations=8, precision="fp64",
                                           tol_max_rel=1e-30, ng_every=ng_every)
    it_cpu, hist = orc.compute_level_populations(use_ng=True, max_iter=8, tol_max_rel=1e-30,
                                                 ng_every=ng_every or 4)
    assert it_gpu == it_cpu == 8
    pop_g = sim.population
    assert rel_err(pop_g, orc.pop, floor=1e-10 * model.population_tot.max()) < FP64_RTOL
    assert np.allclose(sim.error_max, hist, rtol=1e-4, atol=1e-12)


def test_ali_converges_config1_density(gpu):
    """Full ALI + Ng to 1e-4 on the lattice cloud; same iteration count and
    populations as the oracle."""
    model = M.lattice_cloud(10, name="lattice10")
    sim, orc = setup_pair(model, keep_J=False)
    it_gpu = sim.compute_level_populations(True, 200, "fp64", tol_max_rel=1e-4)
    it_cpu, _ = orc.compute_level_populations(True, 200, 1e-4)
    assert sim.converged
    assert abs(it_gpu - it_cpu) <= 1
    assert rel_err(sim.population, orc.pop) < 1e-4


def test_errors_are_status_codes(gpu):
    """A neighbour list with a dead end yields MGR_ERR_TRACE, not a fault."""
    from magritte_b200 import MagritteError
    model = broken_lattice()
    sim = Simulation(model)
    with pytest.raises(MagritteError) as e:
        sim.trace()
    assert e.value.status == 2


@pytest.mark.parametrize("make", [M.config1, lambda: small_wind(10, 5, 7), M.config3,
                                  lambda: M.wind_model(9, seed=3, nlev=4, nside=2, vmax=40e3)])
def test_radiation_field_mixed(gpu, make):
    """Mixed precision against the FP64 oracle: J, Jlin and the ALO to 1e-4."""
    model = make()
    sim, orc = setup_pair(model, keep_J=False)
    sim.compute_radiation_field("mixed", keep_J=True)
    orc.compute_radiation_field()
    orc.compute_Jeff()
    assert rel_err(sim.J, orc.J) < MIXED_RTOL
    assert rel_err(sim.Jlin, orc.Jlin) < MIXED_RTOL
    assert rel_err(sim.Lambda, orc.Ls) < MIXED_RTOL


def test_ali_mixed_populations(gpu):
    """Converged populations in mixed precision against the FP64 oracle."""
    model = M.lattice_cloud(10, name="lattice10")
    sim, orc = setup_pair(model, keep_J=False)
    sim.compute_level_populations(True, 300, "mixed", tol_max_rel=1e-7)
    assert sim.converged
    orc.compute_level_populations(True, 300, 1e-7)
    assert rel_err(sim.population, orc.pop) < MIXED_RTOL


def test_mixed_patches_inverted_lines(gpu):
    """Populations inverted in a block of cells: the mixed solve sends the
    affected (origin, pair, bin) solves to the double-precision patch pass
    and still agrees with the FP64 solve to 1e-4; the FP64 solve agrees with
    the oracle."""
    model = small_wind(10, 5, 7)
    sim, orc = setup_pair(model, keep_J=False)
    pop = sim.population.copy()
    ld = model.linedata
    i, j = int(ld.irad[0]), int(ld.jrad[0])
    g = ld.weight
    # cells 100..399: upper level of line 0 over-populated (n_i/g_i > n_j/g_j)
    cells = slice(100, 400)
    pop[cells, i] = 5.0 * pop[cells, j] * g[i] / g[j]
    pop[cells] *= (model.population_tot[cells] / pop[cells].sum(1))[:, None]
    sim.population = pop
    orc.set_populations(pop)
    sim.compute_radiation_field("fp64", keep_J=True)
    J64, L64 = sim.J.copy(), sim.Lambda.copy()
    orc.compute_radiation_field()
    assert rel_err(J64, orc.J, floor=1e-10 * np.abs(orc.J).max()) < FP64_RTOL
    sim.compute_radiation_field("mixed", keep_J=True)
    patched, fallbacks = sim.patch_stats()
    assert patched > 0 and fallbacks == 0
    assert rel_err(sim.J, J64, floor=1e-6 * np.abs(J64).max()) < MIXED_RTOL
    # a patch list far too small: the origins whose failures overflow it are
    # solved again in double, the rest keeps its float solve and patches
    J_ok, L_ok = sim.J.copy(), sim.Lambda.copy()
    sim.set_patch_capacity(16)
    sim.compute_radiation_field("mixed", keep_J=True)
    patched2, fallbacks2 = sim.patch_stats()
    assert 0 < fallbacks2 < model.ncells
    assert rel_err(sim.J, J64, floor=1e-6 * np.abs(J64).max()) < MIXED_RTOL
    assert rel_err(sim.Lambda, L64, floor=1e-6 * np.abs(L64).max()) < MIXED_RTOL
    # and through the traces rebuilt per batch of origins
    sim.set_trace_budget(1 << 19)
    sim.compute_radiation_field("mixed", keep_J=True)
    assert rel_err(sim.J, J_ok, floor=1e-6 * np.abs(J64).max()) < MIXED_RTOL
    assert rel_err(sim.Lambda, L_ok, floor=1e-6 * np.abs(L64).max()) < MIXED_RTOL


def test_generic_kernels_few_bins(gpu):
    """21 bins per line (a 32-bin chunk spans three lines): the generic FP64
    and mixed kernels run instead of the staged ones; FP64 against the oracle
    to 1e-6, mixed to 1e-4."""
    model = M.lattice_cloud(8, nquads=21, name="lattice8_q21")
    sim, orc = setup_pair(model, keep_J=False)
    sim.compute_radiation_field("fp64", keep_J=True)
    orc.compute_radiation_field()
    orc.compute_Jeff()
    assert sim.tuning("fp64")["kernel"] == "generic"
    assert rel_err(sim.J, orc.J) < FP64_RTOL
    assert rel_err(sim.Lambda, orc.Ls) < FP64_RTOL
    sim.compute_radiation_field("mixed", keep_J=True)
    assert sim.tuning("mixed")["kernel"] == "generic"
    assert rel_err(sim.J, orc.J) < MIXED_RTOL
