"""The partitioned ALI driver (``magritte_b200.partition``) on CPU ranks.

Two (and three) processes joined by a ``gloo`` process group run the
driver's loop -- formal solve of their own origins, statistical equilibrium
of their own cells, all-gather of the population blocks, Ng on every rank --
with a shard backend built on the CPU oracle standing in for the device
(this file only; the product backend is ``DeviceShard`` over the C ABI).
The partitioned run must reproduce the unpartitioned oracle ALI exactly:
same iteration count, same history, bit-identical populations.
"""
import os
import tempfile

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import partition as P

import oracle

TOL = 1e-6


def small_wind():
    return M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8")


class OracleShard:
    """Shard backend over the CPU oracle: the same steps as DeviceShard."""

    def __init__(self, model, rank, world):
        import torch
        self.orc = oracle.Oracle(model).setup()
        self.N, self.nlev = model.ncells, model.linedata.nlev
        self.world = world
        self.begin, self.end = P.shard_bounds(self.N, world)[rank]
        self.pop = torch.from_numpy(self.orc.pop.reshape(-1))   # shares the oracle's array

    def formal_solve(self):
        self.orc.compute_radiation_field(origins=np.arange(self.begin, self.end), nthreads=2)

    def level_local(self):
        # every cell's rate equations (the history shifts for all cells);
        # the other shards' cells are overwritten by the exchange
        self.orc.compute_Jeff()
        oracle.lib().orc_statistical_equilibrium(self.orc.M, self.orc.S)

    def exchange_views(self):
        c = P._chunk(self.N, self.world) * self.nlev
        return [(self.pop, self.begin * self.nlev, self.end * self.nlev, c, self.N * self.nlev)]

    def level_finish(self):
        oracle.lib().orc_check_convergence(self.orc.M, self.orc.S)
        oracle.lib().orc_set_emissivity_opacity(self.orc.M, self.orc.S)

    def ng_step(self):
        self.orc.ng_acceleration()

    def stats(self):
        return (self.orc.fraction_not_converged, self.orc.relative_change_mean,
                self.orc.relative_change_max)


def _rank_main(rank, world, port, out, ng_every=0):
    import torch.distributed as dist
    os.environ["OMP_NUM_THREADS"] = "2"
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        shard = OracleShard(small_wind(), rank, world)
        it, hist, conv = P.partitioned_level_populations(shard, use_ng=True, max_iter=40,
                                                         tol_max_rel=TOL, ng_every=ng_every)
        np.savez(f"{out}_{rank}.npz", it=it, hist=np.array(hist), conv=conv,
                 pop=shard.orc.pop)
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world,ng_every", [(2, 0), (3, 0), (2, 3)])
def test_partitioned_ali_reproduces_unpartitioned(world, ng_every):
    """ng_every = 3: the Ng step after three normal iterations, as the
    oracle's ALI with the same option runs it."""
    import torch.multiprocessing as mp
    model = small_wind()
    ref = oracle.Oracle(model).setup()
    it_ref, hist_ref = ref.compute_level_populations(True, 40, TOL, nthreads=2,
                                                     ng_every=ng_every or 4)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "rank")
        mp.start_processes(_rank_main, args=(world, _free_port(), out, ng_every), nprocs=world,
                           join=True, start_method="spawn")
        res = [np.load(f"{out}_{r}.npz") for r in range(world)]
    for r in res:
        assert bool(r["conv"])
        assert int(r["it"]) == it_ref
        assert np.array_equal(r["hist"], hist_ref)
        assert np.array_equal(r["pop"], ref.pop)


def test_shard_bounds_cover_cells_in_aligned_blocks():
    for n, w in [(262144, 8), (1000, 3), (512, 2), (33, 1)]:
        b = P.shard_bounds(n, w)
        assert b[0][0] == 0 and b[-1][1] == n
        for (b0, e0), (b1, _) in zip(b, b[1:]):
            assert e0 == b1 and b0 % P.CELL_ALIGN == 0
