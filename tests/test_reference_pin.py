"""The C oracle against the reference's own C++ (CPU; test infrastructure).

``oracle/ref_build.sh`` compiles Magritte's CPU path from its unmodified
sources (with a project-written Eigen subset and an OpenMP-only
configure.hpp) into ``oracle/_ref/magritte_ref``, which reads a model folder
in Magritte's text layout (written by ``magritte_b200.io_text``) and runs
the reference's own functions: ``Geometry::trace_ray<CoMoving>``,
``Simulation::compute_radiation_field`` + ``compute_Jeff``, and
``Simulation::compute_level_populations``.  These tests run the C oracle on
the same models and require agreement to 1e-12 relative (bit-exact where
the arithmetic is the same sequence of operations: traces, J, the ALO).

The binary exists only where the reference's sources are present (it is
built next to them); elsewhere the tests skip.
"""
import os
import subprocess

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import io_text

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "magritte_ref")
THREADS = min(8, os.cpu_count() or 1)

needs_ref = pytest.mark.skipif(not os.path.exists(REF),
                               reason="oracle/_ref not built (needs the reference's sources)")


def run_ref(model, tmp_path, *args, pops=None):
    folder = str(tmp_path / "model") + "/"
    out = tmp_path / "out"
    out.mkdir(exist_ok=True)
    io_text.write_model(model, folder)
    if pops is not None:
        io_text.write_populations(folder, pops)
    env = dict(os.environ, OMP_NUM_THREADS=str(THREADS))
    r = subprocess.run([REF, folder, str(out), *args], capture_output=True, text=True, env=env,
                       cwd=str(out),
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    return out


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    return float(np.nanmax(r)) if r.size else 0.0


def small_wind():
    return M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8")


def small_turb():
    return M.turbulent_cloud(5, seed=903, npairs=12, name="turb5")


def inverted_pops(model):
    """LTE populations with line 0 inverted in a block of cells."""
    o = oracle.Oracle(model).setup()
    pop = o.pop.copy()
    ld = model.linedata
    i, j = int(ld.irad[0]), int(ld.jrad[0])
    cells = slice(10, 60)
    pop[cells, i] = 5.0 * pop[cells, j] * ld.weight[i] / ld.weight[j]
    pop[cells] *= (model.population_tot[cells] / pop[cells].sum(1))[:, None]
    return pop


@needs_ref
@pytest.mark.parametrize("make", [M.config1, M.config3, small_wind, small_turb])
def test_radiation_field_matches_reference(tmp_path, make):
    model = make()
    out = run_ref(model, tmp_path, "radiation")
    N, K, nf = model.ncells, model.nlines, model.nfreqs
    orc = oracle.Oracle(model).setup()
    orc.compute_radiation_field(nthreads=THREADS)
    orc.compute_Jeff()
    J = np.fromfile(out / "J.bin").reshape(N, -1)[:, :nf]
    assert rel(J, orc.J) <= 1e-12
    assert rel(np.fromfile(out / "Jlin.bin").reshape(N, K), orc.Jlin) <= 1e-12
    assert rel(np.fromfile(out / "Lambda.bin").reshape(N, K), orc.Ls) <= 1e-12
    assert rel(np.fromfile(out / "population.bin").reshape(N, -1), orc.pop) <= 1e-12


@needs_ref
def test_radiation_field_non_lte_populations_matches_reference(tmp_path):
    """Populations given in the model folder, one line inverted in a block
    of cells (negative line opacities reach the solver)."""
    model = small_wind()
    pop = inverted_pops(model)
    out = run_ref(model, tmp_path, "radiation", "--pops", pops=pop)
    orc = oracle.Oracle(model).setup()
    orc.set_populations(pop)
    orc.compute_radiation_field(nthreads=THREADS)
    orc.compute_Jeff()
    N, K = model.ncells, model.nlines
    J = np.fromfile(out / "J.bin").reshape(N, -1)[:, :model.nfreqs]
    assert rel(J, orc.J) <= 1e-12
    assert rel(np.fromfile(out / "Lambda.bin").reshape(N, K), orc.Ls) <= 1e-12


@needs_ref
@pytest.mark.parametrize("make", [M.config1, small_wind, lambda: M.wind_model(9, seed=3, nlev=4,
                                                                              nside=2, vmax=40e3)])
def test_traces_match_reference(tmp_path, make):
    model = make()
    rng = np.random.default_rng(3)
    origins = rng.choice(model.ncells, size=min(25, model.ncells), replace=False)
    out = run_ref(model, tmp_path, "trace", *[str(int(o)) for o in origins])
    lens = np.fromfile(out / "trace_len.bin", dtype=np.int64)
    cells = np.fromfile(out / "trace_cell.bin", dtype=np.int64)
    sh = np.fromfile(out / "trace_shift.bin")
    dz = np.fromfile(out / "trace_dZ.bin")
    orc = oracle.Oracle(model)
    k = 0
    pos = 0
    for o in origins:
        for r in range(model.nrays):
            c2, s2, z2 = orc.trace_ray(int(o), r)
            n = lens[k]
            k += 1
            assert n == c2.shape[0], (o, r)
            assert np.array_equal(cells[pos:pos + n], c2), (o, r)
            assert np.array_equal(sh[pos:pos + n], s2), (o, r)
            assert np.array_equal(dz[pos:pos + n], z2), (o, r)
            pos += n


@needs_ref
@pytest.mark.parametrize("make,max_iter", [(M.config1, 12), (small_wind, 9)])
def test_level_populations_match_reference(tmp_path, make, max_iter):
    """The reference's ALI loop (Ng after every four iterations, its own
    stop test fraction_not_converged <= 0.005) against the oracle's loop
    stepped the same way: same iteration count, same history of the mean
    relative change (the reference leaves relative_change_max unset), same
    populations."""
    model = make()
    out = run_ref(model, tmp_path, "ali", str(max_iter))
    it_ref = int(np.fromfile(out / "iterations.bin", dtype=np.int64)[0])
    mean_ref = np.fromfile(out / "error_mean.bin")
    orc = oracle.Oracle(model).setup()
    means, normal, it = [], 0, 0
    while it < max_iter:
        it += 1
        if normal == 4:
            orc.ng_acceleration()
            normal = 0
        else:
            orc.compute_radiation_field(nthreads=THREADS)
            orc.compute_Jeff()
            orc.compute_level_populations_from_stateq()
            normal += 1
        means.append(orc.relative_change_mean)
        if not orc.fraction_not_converged > 0.005:
            break
    assert it == it_ref
    # the changes are relative population changes: their rounding floor is
    # absolute (a change of 3e-10 carries the 1e-16 rounding of the LU)
    assert np.allclose(means, mean_ref, rtol=1e-9, atol=1e-13)
    pop = np.fromfile(out / "population.bin").reshape(model.ncells, -1)
    floor = 1e-10 * model.population_tot[:, None]
    mask = orc.pop > floor
    assert rel(pop[mask], orc.pop[mask]) <= 1e-10
    # the oracle's own loop agrees with its stepped form
    orc2 = oracle.Oracle(model).setup()
    it2, _ = orc2.compute_level_populations(True, max_iter, 0.0, nthreads=THREADS)
    assert it2 == it_ref and np.array_equal(orc2.pop, orc.pop)


# ------------------------------------------------------------ model folders

def test_model_folder_round_trip(tmp_path):
    model = M.wind_model(6, seed=5, nlev=6, nside=1, name="wind6")
    folder = str(tmp_path / "m") + "/"
    io_text.write_model(model, folder)
    back = io_text.read_model(folder)
    for f in ("position", "velocity", "nbr_offsets", "nbr_list", "boundary2cell",
              "boundary_temperature", "rays", "ray_weights", "temperature", "vturb2",
              "abundance", "quad_roots", "quad_weights"):
        assert np.array_equal(getattr(back, f), getattr(model, f)), f
    a, b = model.linedata, back.linedata
    assert a.num == b.num and a.inverse_mass == b.inverse_mass
    for f in ("energy", "weight", "irad", "jrad", "A", "frequency", "Bs", "Ba"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert len(a.colpar) == len(b.colpar)
    for ca, cb in zip(a.colpar, b.colpar):
        assert ca.num_col_partner == cb.num_col_partner and ca.orth_or_para_H2 == cb.orth_or_para_H2
        for f in ("icol", "jcol", "tmp", "Cd", "Ce"):
            assert np.array_equal(getattr(ca, f), getattr(cb, f)), f
    assert back.pop_prec == model.pop_prec


def test_population_checkpoint_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    pop = rng.lognormal(size=(50, 7))
    prev = [rng.lognormal(size=(50, 7)) for _ in range(3)]
    folder = str(tmp_path / "c") + "/"
    io_text.write_populations(folder, pop, prev=prev)
    back = io_text.read_populations(folder)
    assert np.array_equal(back["population"], pop)
    for i in range(3):
        assert np.array_equal(back[f"prev{i + 1}"], prev[i])


@needs_ref
@pytest.mark.parametrize("make,ray,width", [(M.config1, 0, 2e-4), (small_wind, 1, 2e-5),
                                            (small_turb, 3, 3e-5)])
def test_image_matches_reference(tmp_path, make, ray, width):
    """compute_and_write_image: rest-frame traces, solve_for_image, the
    emergent intensities at both ends of every cell's ray pair."""
    model = make()
    out = run_ref(model, tmp_path, "image", str(ray), repr(width))
    orc = oracle.Oracle(model).setup()
    orc.compute_spectral_discretisation_image(width)
    I_m, I_p = orc.compute_image(ray, nthreads=THREADS)
    d = str(out) + "/"
    assert rel(I_m, io_text.read_array(d, f"Simulation/Image/I_m_{ray}")) <= 1e-12
    assert rel(I_p, io_text.read_array(d, f"Simulation/Image/I_p_{ray}")) <= 1e-12


def scattering_terms(model, orc):
    """Deterministic U, V of emissivity size (the reference adds U to the
    emissivity): fractions of the line emissivity at each cell's bins,
    varying with pair, cell and bin."""
    KB, AMU, CC = 1.38064852e-23, 1.66053904e-27, 2.99792458e8
    pw = np.sqrt(2.0 * KB / (AMU * CC ** 2) * model.linedata.inverse_mass * model.temperature
                 + model.vturb2)
    nu = orc.nu
    line = model.linedata.frequency
    width = line[None, :] * pw[:, None]
    x = (nu[:, :, None] - line[None, None, :]) / width[:, None, :]
    phi = np.where(np.abs(x) <= 11.0, np.exp(-x * x) / (np.sqrt(np.pi) * width[:, None, :]), 0.0)
    eta = (orc.emissivity[:, None, :] * nu[:, :, None] * phi).sum(-1)
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
    return np.ascontiguousarray(U), np.ascontiguousarray(V)


@needs_ref
@pytest.mark.parametrize("make", [M.config1, small_wind])
def test_scattering_solve_matches_reference(tmp_path, make):
    """setup_using_scattering + solve_using_scattering (never called by the
    reference's own driver) for every ray pair and origin, against the
    oracle's restatement: u and v at the origins and J."""
    model = make()
    orc = oracle.Oracle(model).setup()
    U, V = scattering_terms(model, orc)
    U.tofile(str(tmp_path / "U.bin"))
    V.tofile(str(tmp_path / "V.bin"))
    out = run_ref(model, tmp_path, "scatter", str(tmp_path / "U.bin"), str(tmp_path / "V.bin"))
    u, v = orc.compute_radiation_field_scattering(U, V, nthreads=THREADS)
    shape = u.shape
    ur = np.fromfile(out / "u.bin").reshape(shape)
    vr = np.fromfile(out / "v.bin").reshape(shape)
    assert rel(u, ur) <= 1e-12
    nz = vr != 0
    assert np.array_equal(v == 0, ~nz)
    assert rel(v[nz], vr[nz]) <= 1e-12
    J = np.fromfile(out / "J.bin").reshape(model.ncells, model.nfreqs)
    assert rel(orc.J, J) <= 1e-12
