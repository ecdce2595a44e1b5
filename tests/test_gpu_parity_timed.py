"""Parity of the configurations the benchmark times, against the CPU oracle.

The headline runs the 64^3 wind in mixed precision from the learned warm
start; the north-star model is the 128^3 turbulent cloud (21-level rotor,
41 bins per line, 48 ray pairs) in mixed precision; the batch workload runs
256 winds of a 20-level rotor as one point cloud.  These tests check each
of those set-ups against the oracle (the reference's algorithm restated in
C, FP64), not against the device's own FP64 path:

* 64^3 wind: Jlin and the ALO at sampled origins, mixed precision, at the
  LTE populations and at the learned warm start's populations (1e-4), and
  FP64 at the warm start (1e-6).
* turbulent cloud of the 128^3 family at 12^3: the same at sampled origins;
  at 8^3 the full ALI + Ng to convergence in FP64 (1e-6 after the same
  number of iterations) and in mixed precision (1e-4).
* three members of the 256-model batch solved inside one batch: each
  member's converged populations and iteration count against the oracle's
  ALI of that member alone (FP64 1e-6, mixed 1e-4).

Tolerances: 1e-6 relative in FP64, 1e-4 in mixed precision.  Converged
populations are compared at 1e-6 (FP64) on levels holding more than 1e-6 of
the cell's total; levels between 1e-10 (the reference's convergence cut)
and 1e-6 of the total are compared at 1e-4, because the per-cell LU solves
of the device and the oracle round differently and a level at 1e-9 of the
total carries the absolute rounding of the whole solution (about
cond * 1e-16 of the largest population), i.e. ~1e-6 of itself.
"""
import os

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation

import oracle

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6
MIXED_RTOL = 1e-4
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "magritte_b200", "weights")
THREADS = os.cpu_count() or 1


def rel_err(a, b, mask=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    if mask is not None:
        r = r[mask]
    return float(np.nanmax(r)) if r.size else 0.0


def device(model):
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    return sim


def check_sampled(sim, model, origins, pop, precision, rtol):
    """One formal solve of the device at populations `pop` against the
    oracle's solve of the sampled origins at the same populations."""
    sim.population = pop
    sim.compute_radiation_field(precision)
    orc = oracle.Oracle(model).setup()
    orc.set_populations(pop)
    orc.compute_radiation_field(origins=origins, nthreads=THREADS)
    assert orc.trace_errors == 0
    orc.compute_Jeff()
    e_j = rel_err(sim.Jlin[origins], orc.Jlin[origins])
    e_l = rel_err(sim.Lambda[origins], orc.Ls[origins])
    assert e_j < rtol, (precision, e_j)
    assert e_l < rtol, (precision, e_l)
    return e_j, e_l


def check_populations(got, ref, model, rtol):
    """rtol on levels above 1e-6 of the total (FP64 rounding of the rate
    solves bounds the rest); 1e-4 on every level above 1e-10 of it."""
    tot = model.population_tot[:, None]
    big = ref > 1e-6 * tot
    small = ref > 1e-10 * tot
    e_big = rel_err(got, ref, big)
    e_all = rel_err(got, ref, small)
    assert e_big < rtol, ("levels > 1e-6 n_tot", e_big)
    assert e_all < max(rtol, MIXED_RTOL), ("levels > 1e-10 n_tot", e_all)


def warm_start_pops(sim, weights):
    from magritte_b200.learned import WarmStartNet
    net = WarmStartNet.load(os.path.join(WEIGHTS, weights))
    sim.warm_start(net)
    return sim.population


# ------------------------------------------------------------ 64^3 wind

def test_wind64_mixed_and_learned_start_vs_oracle(gpu):
    model = M.config2()
    sim = device(model)
    sim.compute_LTE_level_populations()
    lte = sim.population
    rng = np.random.default_rng(21)
    origins = np.sort(rng.choice(model.ncells, size=48, replace=False))
    check_sampled(sim, model, origins, lte, "mixed", MIXED_RTOL)
    warm = warm_start_pops(sim, "wind_rotor10.npz")
    assert not np.allclose(warm, lte)
    check_sampled(sim, model, origins, warm, "mixed", MIXED_RTOL)
    check_sampled(sim, model, origins, warm, "fp64", FP64_RTOL)


# ---------------------------------------------- 128^3 turbulent-cloud family

def test_turbulent_family_formal_solve_vs_oracle(gpu):
    """21-level rotor, 20 lines x 41 bins, 48 ray pairs, Doppler
    sub-points on the rays, at 12^3: LTE and learned-start populations."""
    model = M.turbulent_cloud(12, seed=901, name="turb12")
    assert model.nfreqs == 820 and model.nrays == 96 and model.linedata.nlev == 21
    sim = device(model)
    sim.compute_LTE_level_populations()
    lte = sim.population
    rng = np.random.default_rng(5)
    origins = np.sort(rng.choice(model.ncells, size=48, replace=False))
    check_sampled(sim, model, origins, lte, "fp64", FP64_RTOL)
    check_sampled(sim, model, origins, lte, "mixed", MIXED_RTOL)
    warm = warm_start_pops(sim, "turb_rotor21.npz")
    check_sampled(sim, model, origins, warm, "mixed", MIXED_RTOL)
    assert sim.tuning("mixed")["kernel"] == "staged"


@pytest.fixture(scope="module")
def turb8_oracle():
    """The oracle's full ALI + Ng on an 8^3 cloud of the family, to a max
    relative change below 1e-5 (11 iterations).  Below about 3e-7 this
    cloud's local-ALO + Ng iteration stalls and wanders (its max change
    stays between 1e-7 and 3e-7 for ten more iterations in the oracle
    itself), so the iteration count to a tighter tolerance is not a stable
    property of the algorithm."""
    model = M.turbulent_cloud(8, seed=902, name="turb8")
    orc = oracle.Oracle(model).setup()
    it, hist = orc.compute_level_populations(True, 40, 1e-5, nthreads=THREADS)
    assert hist[-1] < 1e-5
    return model, it, hist, orc.pop.copy()


def test_turbulent_family_converged_fp64_vs_oracle(gpu, turb8_oracle):
    model, it_cpu, hist, pop_cpu = turb8_oracle
    sim = device(model)
    sim.compute_LTE_level_populations()
    it = sim.compute_level_populations(True, 40, "fp64", tol_max_rel=1e-5)
    assert sim.converged and it == it_cpu
    check_populations(sim.population, pop_cpu, model, FP64_RTOL)
    assert np.allclose(sim.error_max, hist, rtol=1e-4, atol=1e-9)


def test_turbulent_family_converged_mixed_vs_oracle(gpu, turb8_oracle):
    model, it_cpu, _, pop_cpu = turb8_oracle
    sim = device(model)
    sim.compute_LTE_level_populations()
    sim.compute_level_populations(True, 40, "mixed", tol_max_rel=1e-5, use_graph=True)
    assert sim.converged
    check_populations(sim.population, pop_cpu, model, MIXED_RTOL)


# ------------------------------------------------------ 256-model batch

BATCH_MEMBERS = (30, 146, 122)   # three of the smallest members (about 2k points each)


@pytest.fixture(scope="module")
def batch_oracle():
    """Each member alone through the oracle's ALI to 1e-5 (tighter targets
    reach the region where the Ng coefficients are ill-conditioned and
    last-bit differences change the trajectory, as for the cloud above)."""
    out = []
    for m in BATCH_MEMBERS:
        model = M.config4_member(m)
        orc = oracle.Oracle(model).setup()
        it, _ = orc.compute_level_populations(True, 100, 1e-5, nthreads=THREADS)
        out.append((model, it, orc.pop.copy()))
    return out


@pytest.mark.parametrize("precision,rtol", [("fp64", FP64_RTOL), ("mixed", MIXED_RTOL)])
def test_batch_members_vs_oracle(gpu, batch_oracle, precision, rtol):
    batch = M.concat_models([m for m, _, _ in batch_oracle], name="batch3")
    sim = device(batch)
    sim.compute_LTE_level_populations()
    sim.compute_level_populations(True, 100, precision, tol_max_rel=1e-5, use_graph=True)
    assert sim.converged
    _, iters = sim.segment_results()
    pop = sim.population
    seg = batch.meta["segments"]
    for s, (model, it_cpu, pop_cpu) in enumerate(batch_oracle):
        if precision == "fp64":
            assert iters[s] == it_cpu, (s, iters[s], it_cpu)
        else:
            assert abs(iters[s] - it_cpu) <= 2, (s, iters[s], it_cpu)
        check_populations(pop[seg[s]:seg[s + 1]], pop_cpu, model, rtol)
