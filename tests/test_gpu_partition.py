"""Shards of a partitioned run through the C ABI, on one GPU.

Two Simulation handles own the two halves of the origins of one model
(``mgr_set_origin_range``).  They take the steps of the partitioned driver
one after the other in this process -- formal solve of their origins,
statistical equilibrium of their cells (``mgr_stateq_local``), exchange of
population blocks and convergence partials (device copies here; an NCCL
all-gather between GPUs), ``mgr_stateq_finish`` -- and must reproduce the
unpartitioned FP64 run bit for bit.  No kernel of one handle waits on the
other's: the exchange happens between launches, on the host's order.
"""
import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import Simulation
from magritte_b200 import partition as P

pytestmark = pytest.mark.gpu

TOL = 1e-6


def setup(model):
    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    return sim


def exchange_local(shards):
    """What all_gather_blocks does across ranks, for shards in one process."""
    import torch
    nviews = len(shards[0].exchange_views())
    for v in range(nviews):
        parts = []
        for s in shards:
            t, lo, hi, _, _ = s.exchange_views()[v]
            parts.append(t[lo:hi].clone())
        full = torch.cat(parts)
        for s in shards:
            t, _, _, _, n = s.exchange_views()[v]
            t[:n].copy_(full[:n])
    torch.cuda.synchronize()


def run_shards(model, world, max_iter=40, tol=TOL):
    sims = [setup(model) for _ in range(world)]
    shards = [P.DeviceShard(s, k, world, "fp64") for k, s in enumerate(sims)]
    it, normal, hist, more = 0, 0, [], True
    while more and it < max_iter:
        it += 1
        if normal == 4:
            for s in shards:
                s.ng_step()
            normal = 0
        else:
            for s in shards:
                s.formal_solve()
                s.level_local()
            exchange_local(shards)
            for s in shards:
                s.level_finish()
            normal += 1
        stats = [s.stats() for s in shards]
        assert all(st == stats[0] for st in stats)
        hist.append(stats[0][2])
        more = not stats[0][2] < tol
    return it, hist, [s.population for s in sims]


@pytest.mark.parametrize("world", [2, 3])
def test_device_shards_reproduce_unpartitioned_run(gpu, world):
    model = M.wind_model(10, seed=7, nlev=5, nside=1, name="wind10")
    whole = setup(model)
    it = whole.compute_level_populations(True, 40, "fp64", tol_max_rel=TOL)
    assert whole.converged
    it_s, hist_s, pops = run_shards(model, world)
    assert it_s == it
    assert np.array_equal(np.array(hist_s), np.array(whole.error_max))
    for p in pops:
        assert np.array_equal(p, whole.population)


def test_origin_range_is_validated(gpu):
    from magritte_b200 import MagritteError
    model = M.wind_model(6, seed=7, nlev=4, nside=1, name="wind6")
    sim = setup(model)
    with pytest.raises(MagritteError):
        sim.set_origin_range(3, 100)          # not a multiple of 4
    with pytest.raises(MagritteError):
        sim.set_origin_range(0, model.ncells + 4)
    sim.set_origin_range(0, 100)
    with pytest.raises(MagritteError):        # the unpartitioned loop refuses a shard
        sim.compute_level_populations(True, 5, "fp64")
