"""The allocation-free convergence entry point, through the C ABI.

mgr_convergence_noalloc serves callers that cannot allocate device memory
(applications that reserve all GPU memory in their own pool and forbid
cudaMalloc).  The test owns every device buffer (allocated here with torch,
standing in for such a caller's pool), calls the entry point twice in a row,
and compares both results with the handle-based path's statistics for the
same populations.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation, _capi

pytestmark = pytest.mark.gpu


def test_convergence_noalloc_matches_handle_path(gpu):
    import torch
    model = M.wind_model(10, seed=7, nlev=5, nside=1, name="noalloc_wind10")
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    sim.compute_radiation_field("fp64")
    sim.compute_Jeff()
    before = sim.population
    sim.compute_level_populations_from_stateq()
    after = sim.population
    fnc, rcm, mx = sim.convergence()
    sim.close()

    dev = torch.device("cuda", 0)
    pop = torch.tensor(after, dtype=torch.float64, device=dev).contiguous()
    prev = torch.tensor(before, dtype=torch.float64, device=dev).contiguous()
    tot = torch.tensor(model.population_tot, dtype=torch.float64, device=dev).contiguous()
    stats = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    lib = _capi.load()
    for _ in range(2):
        stats.fill_(float("nan"))
        st = lib.mgr_convergence_noalloc(pop.data_ptr(), prev.data_ptr(), tot.data_ptr(),
                                         model.ncells, model.linedata.nlev, model.pop_prec,
                                         stats.data_ptr(), None)
        assert st == 0
        torch.cuda.synchronize()
        got = stats.cpu().numpy()
        assert abs(got[0] - fnc) <= 1e-12
        assert abs(got[1] - rcm) <= 1e-12 * max(rcm, 1e-300)
        assert got[2] == mx


def test_convergence_noalloc_rejects_oversize(gpu):
    lib = _capi.load()
    big = _capi.NOALLOC_MAX_ELEMENTS // 2 + 1
    # checked before any device access: the pointers are never read
    fake = C.c_void_p(16)
    st = lib.mgr_convergence_noalloc(fake, fake, fake, big, 2, 1e-6, fake, None)
    assert st == 10   # MGR_ERR_TOO_LARGE
    st = lib.mgr_convergence_noalloc(None, fake, fake, 10, 2, 1e-6, fake, None)
    assert st == 1    # MGR_ERR_INVALID_ARG


def _numpy_convergence(pop, prev, tot, nlev, pop_prec):
    """check_for_convergence (lineProducingSpecies.tpp:120-171) restated in
    numpy: count, mean and max of 2|n - n'|/(n + n') over levels with
    n > 1e-10 n_tot."""
    a = pop.reshape(-1)
    b = prev.reshape(-1)
    keep = a > 1.0e-10 * np.repeat(tot, nlev)
    rc = 2.0 * np.abs(a - b)
    rc = rc / (a + b)
    rc = np.where(keep, rc, 0.0)
    n = a.size
    return float(np.count_nonzero(rc > pop_prec)) / n, float(rc.sum()) / n, float(rc.max())


@pytest.mark.parametrize("ncells,nlev", [(400_000, 3), (16_777_216, 4)])
def test_convergence_noalloc_large(gpu, ncells, nlev):
    """More than 1024 first-pass blocks (the final pass loops over the
    partials), and exactly MGR_NOALLOC_MAX_ELEMENTS cell-levels (65,536
    blocks, the whole scratch array), on synthetic device arrays."""
    import torch
    assert ncells * nlev > 1_048_576
    rng = np.random.default_rng(ncells)
    prev = rng.lognormal(0.0, 3.0, size=(ncells, nlev))
    pop = prev * (1.0 + rng.normal(0.0, 1e-3, size=prev.shape))
    pop[rng.random(size=pop.shape) < 1e-3] *= 1e-12      # below 1e-10 n_tot: skipped
    tot = pop.sum(axis=1)
    ref = _numpy_convergence(pop, prev, tot, nlev, 1e-4)
    dev = torch.device("cuda", 0)
    tp = torch.from_numpy(pop).to(dev)
    tq = torch.from_numpy(prev).to(dev)
    tt = torch.from_numpy(tot).to(dev)
    stats = torch.empty(3, dtype=torch.float64, device=dev)
    lib = _capi.load()
    for _ in range(2):
        stats.fill_(float("nan"))
        st = lib.mgr_convergence_noalloc(tp.data_ptr(), tq.data_ptr(), tt.data_ptr(), ncells,
                                         nlev, 1e-4, stats.data_ptr(), None)
        assert st == 0
        torch.cuda.synchronize()
        got = stats.cpu().numpy()
        assert got[0] == pytest.approx(ref[0], rel=1e-12, abs=0.0)
        assert got[1] == pytest.approx(ref[1], rel=1e-11)
        assert got[2] == ref[2]
    del tp, tq, tt
    torch.cuda.empty_cache()
