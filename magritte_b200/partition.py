"""ALI iteration partitioned over ranks: one GPU per shard of origins.

The reference splits the ray directions over its MPI ranks and then sums J
(``MPI_reduce_J``, ``src/Model/Radiation/radiation.cpp:292-325``) and
gathers the ALO (``Lambda::MPI_gather``,
``src/Model/Lines/LineProducingSpecies/Lambda/lambda.tpp:191-317``) in every
iteration.  Here the units of work are origins: rank k owns the cells
``bounds[k] = [b_k, e_k)`` (contiguous blocks, multiples of 32 cells).  Per
normal iteration each rank

1. solves the formal problem for its own origins only (Jlin and the ALO of
   its own cells, all ray pairs, every bin);
2. solves the statistical equilibrium of its own cells (Jeff, the rate
   equations), shifting the population history of every cell;
3. all-gathers the new populations of every block and the blocks'
   convergence partials (one collective of ``ncells*nlev + 3*ncells/4``
   doubles over NCCL/NVLink);
4. recomputes emissivities/opacities and the convergence statistics of all
   cells from the gathered arrays.

An Ng step needs no exchange: after step 3 every rank holds the same
populations and history, so each rank runs the same Ng step on all cells.
Because each cell's J, ALO and rate equations are computed on exactly one
rank by the same kernels, and the convergence partials are reduced in the
global block order, an FP64 run on any number of ranks gives the populations
of the unpartitioned run bit for bit.

The driver works on a *shard backend*; :class:`DeviceShard` is the one over
the C ABI (``mgr_set_origin_range``, ``mgr_stateq_local``,
``mgr_stateq_finish``, ``mgr_get_device_buffer``), exchanging device arrays
in place with ``torch.distributed`` (NCCL between GPUs).  Every rank takes
the same collective steps in the same order.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

CELL_ALIGN = 32


def shard_bounds(ncells: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous cell blocks of equal size (a multiple of 32) per rank; the
    last may be shorter, and trailing ranks may own nothing when the model
    is tiny."""
    chunk = CELL_ALIGN * math.ceil(ncells / world / CELL_ALIGN)
    return [(min(ncells, k * chunk), min(ncells, (k + 1) * chunk)) for k in range(world)]


def _chunk(ncells: int, world: int) -> int:
    return CELL_ALIGN * math.ceil(ncells / world / CELL_ALIGN)


class _DeviceArray:
    """A raw device buffer of the library, seen by torch without a copy."""

    def __init__(self, ptr: int, n: int, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def device_tensor(sim, which: int):
    """torch view (float64, 1-D) of one of a Simulation's device arrays."""
    import ctypes as C
    import torch
    from . import _capi
    ptr = C.c_void_p()
    n = C.c_int64()
    sim._ck(sim._lib.mgr_get_device_buffer(sim._h, which, C.byref(ptr), C.byref(n)))
    return torch.as_tensor(_DeviceArray(ptr.value, n.value), device=f"cuda:{sim.device}")


class DeviceShard:
    """Shard backend over a :class:`magritte_b200.Simulation` on one GPU."""

    def __init__(self, sim, rank: int, world: int, precision: str = "fp64",
                 use_graph: bool = False):
        from . import _capi
        self.sim, self.rank, self.world = sim, rank, world
        self.precision = precision
        self.N = sim.model.ncells
        self.nlev = sim.model.linedata.nlev
        self.bounds = shard_bounds(self.N, world)
        b, e = self.bounds[rank]
        if e <= b:
            raise ValueError(f"{world} shards of {self.N} cells leave rank {rank} without cells")
        self.begin, self.end = b, e
        sim.set_origin_range(b, e)
        self.pop = device_tensor(sim, _capi.BUF_POPULATION)
        self.partials = device_tensor(sim, _capi.BUF_PARTIALS)
        self._cells_per_partial = _capi.CELLS_PER_PARTIAL

    # --- one normal iteration, before and after the exchange
    def formal_solve(self):
        self.sim.compute_radiation_field(self.precision)

    def level_local(self):
        self.sim.stateq_local()

    def exchange_views(self):
        """(own slice, full array) pairs in cell-block order."""
        c, nl, cpp = _chunk(self.N, self.world), self.nlev, self._cells_per_partial
        return [(self.pop, self.begin * nl, self.end * nl, c * nl, self.N * nl),
                (self.partials, 3 * (self.begin // cpp), 3 * (-(-self.end // cpp)), 3 * (c // cpp),
                 3 * (-(-self.N // cpp)))]

    def level_finish(self):
        self.sim.stateq_finish()

    def ng_step(self):
        self.sim.ng_acceleration()

    def stats(self):
        return self.sim.convergence()


def all_gather_blocks(views, group=None):
    """All-gathers every rank's own slice of each array into the full array
    (in place).  views: (tensor, own_lo, own_hi, chunk, full_len) with the
    slices in rank order and every rank's chunk the same size."""
    import torch
    import torch.distributed as dist
    for t, lo, hi, chunk, full in views:
        world = dist.get_world_size(group)
        send = torch.zeros(chunk, dtype=t.dtype, device=t.device)
        if hi > lo:
            send[: hi - lo].copy_(t[lo:hi])
        out = torch.empty(world * chunk, dtype=t.dtype, device=t.device)
        dist.all_gather_into_tensor(out, send, group=group)
        t[:full].copy_(out[:full])
    if views and views[0][0].is_cuda:
        # the library's own stream reads these arrays next
        torch.cuda.current_stream(views[0][0].device).synchronize()


def partitioned_level_populations(shard, group=None, use_ng: bool = True, max_iter: int = 1000,
                                  tol_max_rel: float = 0.0,
                                  ng_every: int = 0) -> Tuple[int, List[float], bool]:
    """The ALI loop of ``Simulation::compute_level_populations``
    (``src/Simulation/sim_lines.tpp:61-164``) over the shards of a process
    group: Ng after every ``ng_every`` normal iterations (0: the
    reference's four), stop at max relative change < tol_max_rel (or, with
    tol_max_rel <= 0, the reference's fraction_not_converged <= 0.005).
    Returns (iterations, max relative change of every iteration,
    converged); every rank returns the same."""
    if ng_every != 0 and ng_every < 3:
        raise ValueError("ng_every must be 0 (the reference's 4) or >= 3")
    every = ng_every or 4
    iteration, normal = 0, 0
    hist: List[float] = []
    more = True
    while more and iteration < max_iter:
        iteration += 1
        if use_ng and normal == every:
            shard.ng_step()
            normal = 0
        else:
            shard.formal_solve()
            shard.level_local()
            all_gather_blocks(shard.exchange_views(), group)
            shard.level_finish()
            normal += 1
        fnc, _, mx = shard.stats()
        hist.append(mx)
        more = not (mx < tol_max_rel) if tol_max_rel > 0 else fnc > 0.005
    return iteration, hist, not more
