"""``Simulation``: the reference's Python-facing interface over the C ABI.

Method names and their meaning follow ``magritte.core.Simulation``
(``src/bindings/pyBindings.cpp:404-449``): a user calls

    sim = Simulation(model)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    sim.compute_radiation_field()            # or compute_level_populations()

as in ``tests/integration/test_0_1D_all_constant.py:64-99``.  Every call goes
to hand-written sm_100a kernels through ``libmagritte_b200.so``; errors come
back as :class:`MagritteError` with the C status code.  Differences from the
reference: the model is passed as a :class:`magritte_b200.model.Model`
instead of an ``Io`` object, and ``compute_level_populations`` takes the
options that the ``Io`` overloads fix (Ng, iteration cap) plus the
precision and an optional max-relative-change tolerance.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _capi
from ._capi import MagritteError, MGR_FP64, MGR_MIXED

_PREC = {"fp64": MGR_FP64, "mixed": MGR_MIXED, MGR_FP64: MGR_FP64, MGR_MIXED: MGR_MIXED}


class Simulation:
    def __init__(self, model=None, device: int = 0):
        self._lib = _capi.load()
        h = C.c_void_p()
        st = self._lib.mgr_create(device, C.byref(h))
        if st != 0:
            raise MagritteError(st, "mgr_create failed (no CUDA device?)")
        self._h = h
        self.device = device
        self.model = None
        self.n_off_diag = 0
        self.error_max = []
        self.error_mean = []
        self.fraction_not_converged = []
        if model is not None:
            self.read(model)

    # ------------------------------------------------------------ plumbing
    def _ck(self, st: int):
        if st != 0 and st != 4:
            raise MagritteError(st, self._lib.mgr_last_error(self._h).decode())
        return st

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.mgr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --------------------------------------------------------------- model
    def read(self, model):
        """Uploads the model (replaces ``Model::read(io)``)."""
        desc, keep = _capi.make_desc(model)
        self._ck(self._lib.mgr_upload_model(self._h, C.byref(desc)))
        self.model = model
        seg = model.meta.get("segments") if isinstance(model.meta, dict) else None
        if seg is not None and len(seg) > 2:
            b = np.ascontiguousarray(seg, dtype=np.int64)
            self._ck(self._lib.mgr_set_segments(self._h, b.shape[0] - 1, _capi.ptr(b)))
        return 0

    def set_trace_budget(self, nbytes: int):
        self._ck(self._lib.mgr_set_trace_budget(self._h, int(nbytes)))

    # ---------------------------------------------------- reference calls
    def compute_spectral_discretisation(self) -> int:
        return self._ck(self._lib.mgr_compute_spectral_discretisation(self._h))

    def compute_boundary_intensities(self) -> int:
        return self._ck(self._lib.mgr_compute_boundary_intensities(self._h))

    def compute_LTE_level_populations(self) -> int:
        return self._ck(self._lib.mgr_compute_LTE_level_populations(self._h))

    def compute_radiation_field(self, precision="fp64", keep_J: Optional[bool] = None) -> int:
        if keep_J is not None:
            self._ck(self._lib.mgr_set_keep_J(self._h, int(bool(keep_J))))
        return self._ck(self._lib.mgr_compute_radiation_field(self._h, _PREC[precision]))

    def compute_Jeff(self):
        self._ck(self._lib.mgr_compute_Jeff(self._h))

    def compute_level_populations_from_stateq(self):
        self._ck(self._lib.mgr_compute_level_populations_from_stateq(self._h))
        self._record()

    def ng_acceleration(self):
        self._ck(self._lib.mgr_ng_acceleration(self._h))
        self._record()

    def compute_level_populations(self, use_Ng: bool = True, max_niterations: int = 1000,
                                  precision="fp64", tol_max_rel: float = 0.0,
                                  use_graph: bool = False, ng_every: int = 0) -> int:
        """ALI loop (``Simulation::compute_level_populations``,
        ``sim_lines.tpp:61-164``); returns the iteration count.
        ``tol_max_rel`` > 0 stops at max relative population change < tol;
        ``use_graph`` replays each iteration's launches as CUDA graphs;
        ``ng_every`` is the number of normal iterations before each Ng step
        (0: the reference's 4; at least 3).  For a batch of models every
        model iterates to its own convergence and the count is the batch's
        (``segment_results`` has each model's)."""
        o = _capi.AliOpts()
        o.use_ng = int(bool(use_Ng))
        o.precision = _PREC[precision]
        o.max_iter = int(max_niterations)
        o.tol_max_rel = float(tol_max_rel)
        o.use_graph = int(bool(use_graph))
        o.ng_every = int(ng_every)
        it = C.c_int64(0)
        hist = np.zeros(max(1, int(max_niterations)))
        st = self._ck(self._lib.mgr_compute_level_populations(self._h, C.byref(o), C.byref(it),
                                                              _capi.ptr(hist)))
        self.error_max = list(hist[: it.value])
        self.converged = (st == 0)
        return int(it.value)

    # ------------------------------------------------------ scattering
    def _scat_shape(self):
        m = self.model
        return (m.nrays // 2, m.ncells, m.nfreqs)

    def set_scattering_terms(self, U=None, V=None):
        """Scattering terms U, V [nrays/2, ncells, nfreqs] (None: zeros)."""
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64).reshape(self._scat_shape())
                for a in (U, V)]
        self._ck(self._lib.mgr_set_scattering_terms(
            self._h, *[None if a is None else _capi.ptr(a) for a in arrs]))

    def scattering_terms(self):
        U, V = np.zeros(self._scat_shape()), np.zeros(self._scat_shape())
        self._ck(self._lib.mgr_get_scattering_terms(self._h, _capi.ptr(U), _capi.ptr(V)))
        return U, V

    def compute_radiation_field_scattering(self, keep_J: Optional[bool] = None) -> int:
        """The formal solve with scattering terms
        (``setup_using_scattering`` + ``solve_using_scattering``)."""
        if keep_J is not None:
            self._ck(self._lib.mgr_set_keep_J(self._h, int(bool(keep_J))))
        return self._ck(self._lib.mgr_compute_radiation_field_scattering(self._h))

    def scattering_uv(self):
        """u and v at the origins of the last scattering solve."""
        u, v = np.zeros(self._scat_shape()), np.zeros(self._scat_shape())
        self._ck(self._lib.mgr_get_scattering_uv(self._h, _capi.ptr(u), _capi.ptr(v)))
        return u, v

    def calc_U_and_V(self):
        """Next scattering terms from the last solve (``Radiation::calc_U_and_V``)."""
        self._ck(self._lib.mgr_calc_U_and_V(self._h))

    # ---------------------------------------------------------- images
    def compute_image(self, ray: int, width: float) -> dict:
        """Image along ``ray`` (``Simulation::compute_and_write_image``):
        the image grid ``nu`` [nfreqs], emergent intensities ``I_m``/``I_p``
        [ncells, nfreqs] through the front / end of each cell's ray pair,
        and the image-plane coordinates ``ImX``/``ImY`` [ncells]."""
        m = self.model
        out = {"nu": np.zeros(m.nfreqs), "I_m": np.zeros((m.ncells, m.nfreqs)),
               "I_p": np.zeros((m.ncells, m.nfreqs)), "ImX": np.zeros(m.ncells),
               "ImY": np.zeros(m.ncells)}
        self._ck(self._lib.mgr_compute_image(self._h, int(ray), float(width),
                                             *[_capi.ptr(out[k]) for k in
                                               ("nu", "I_m", "I_p", "ImX", "ImY")]))
        return out

    # ----------------------------------------------------- checkpoints
    def population_history(self):
        """(prev1, prev2, prev3): the iterates Ng acceleration reads."""
        m = self.model
        out = [np.zeros((m.ncells, m.linedata.nlev)) for _ in range(3)]
        self._ck(self._lib.mgr_get_population_history(self._h, *[_capi.ptr(a) for a in out]))
        return tuple(out)

    def set_population_history(self, pop, prev1=None, prev2=None, prev3=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (pop, prev1, prev2, prev3)]
        self._ck(self._lib.mgr_set_population_history(
            self._h, *[_capi.ptr(a) if a is not None else None for a in arrs]))

    def write_checkpoint(self, folder: str, tag: str = ""):
        """Populations and their history in Magritte's text layout
        (``population<tag>``, ``population_prev1..3``, ``J_lin<tag>``,
        ``J_eff<tag>`` of ``Lines/LineProducingSpecies_0/``)."""
        from . import io_text
        io_text.write_populations(folder, self.population, prev=self.population_history(),
                                  Jlin=self.Jlin, Jeff=self.Jeff, tag=tag)

    def read_checkpoint(self, folder: str, tag: str = ""):
        """Restores what write_checkpoint (or the reference's
        LineProducingSpecies::write) stored; the next
        compute_level_populations continues where that run stopped."""
        from . import io_text
        d = io_text.read_populations(folder, tag)
        self.set_population_history(d["population"], d.get("prev1"), d.get("prev2"),
                                    d.get("prev3"))

    # -------------------------------------------------- partitioned runs
    def set_origin_range(self, begin: int, end: int):
        """This handle solves origins (cells) [begin, end) only: one shard of
        a run partitioned over GPUs (``magritte_b200.partition``)."""
        self._ck(self._lib.mgr_set_origin_range(self._h, int(begin), int(end)))

    def stateq_local(self):
        """Jeff and statistical equilibrium of the shard's own cells."""
        self._ck(self._lib.mgr_stateq_local(self._h))

    def stateq_finish(self):
        """Emissivities/opacities and convergence statistics after the
        shards exchanged their populations and partials."""
        self._ck(self._lib.mgr_stateq_finish(self._h))

    # ------------------------------------------------------ model batches
    def segment_results(self):
        """Per-model (fraction not converged, mean, max relative change) at
        each model's last iteration, and the iteration it converged at."""
        n = len(self.model.meta["segments"]) - 1
        st = np.zeros((n, 3))
        it = np.zeros(n, dtype=np.int64)
        self._ck(self._lib.mgr_get_segment_results(self._h, _capi.ptr(st), _capi.ptr(it)))
        return st, it

    def patch_stats(self):
        """(solves of the last mixed formal solve redone in double, mixed
        solves redone entirely in double so far)."""
        a, b = C.c_int64(0), C.c_int64(0)
        self._ck(self._lib.mgr_get_patch_stats(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def set_n_off_diag(self, n_off_diag: int):
        """``parameters.n_off_diag``: 0 or 1 keep the diagonal ALO; M >= 2
        keep the M-1 nearest off-diagonal elements on each side of every ray
        pair and solve the rate equations of all cells as one system."""
        self._ck(self._lib.mgr_set_n_off_diag(self._h, int(n_off_diag)))
        self.n_off_diag = int(n_off_diag)

    def alo_nonlocal(self):
        """The off-diagonal ALO elements of the last formal solve:
        (Loff [N, nrad, nrays/2, 2, M-1], Loff_nr [N, nrays/2, 2, M-1])."""
        m, M1 = self.model, self.n_off_diag - 1
        Loff = np.zeros((m.ncells, m.nlines, m.nrays // 2, 2, M1))
        nr = np.zeros((m.ncells, m.nrays // 2, 2, M1), dtype=np.int64)
        self._ck(self._lib.mgr_get_alo_nonlocal(self._h, _capi.ptr(Loff), _capi.ptr(nr)))
        return Loff, nr

    def nonlocal_sweeps(self) -> int:
        n = C.c_int64()
        self._ck(self._lib.mgr_get_nonlocal_sweeps(self._h, C.byref(n)))
        return n.value

    def set_patch_capacity(self, entries: int):
        """Capacity of the mixed solve's list of solves redone in double
        (0: automatic); origins whose failures overflow it are re-solved in
        double."""
        self._ck(self._lib.mgr_set_patch_capacity(self._h, int(entries)))

    # ------------------------------------------------------------ tuning
    def set_autotune(self, mode=True):
        """True / 1: tune the solve kernel (reusing this process's results
        for the same shape); 2: always re-time; False / 0: off."""
        self._ck(self._lib.mgr_set_autotune(self._h, int(mode)))

    def tuning(self, precision="mixed") -> dict:
        t = _capi.Tuning()
        self._ck(self._lib.mgr_get_tuning(self._h, _PREC[precision], C.byref(t)))
        return {"kernel": {-1: None, 0: "generic", 1: "staged"}[t.kernel],
                "min_blocks": t.min_blocks, "warps_per_block": t.warps_per_block,
                "tuned": bool(t.tuned), "ms": [float(x) for x in t.ms[:3]]}

    def get_npoints_on_rays_comoving(self) -> np.ndarray:
        m = self.model
        out = np.zeros((m.nrays // 2, m.ncells), dtype=np.int64)
        self._ck(self._lib.mgr_get_npoints_on_rays(self._h, _capi.ptr(out)))
        return out

    get_npoints_on_rays = get_npoints_on_rays_comoving

    # --------------------------------------------------------- accessors
    def trace(self):
        self._ck(self._lib.mgr_trace(self._h))

    def trace_ray(self, o: int, r: int):
        n = C.c_int64(0)
        self._ck(self._lib.mgr_get_trace(self._h, o, r, 0, None, None, None, C.byref(n)))
        cap = max(1, n.value)
        cell = np.zeros(cap, dtype=np.int64)
        shift = np.zeros(cap)
        dZ = np.zeros(cap)
        self._ck(self._lib.mgr_get_trace(self._h, o, r, cap, _capi.ptr(cell), _capi.ptr(shift),
                                         _capi.ptr(dZ), C.byref(n)))
        return cell[: n.value], shift[: n.value], dZ[: n.value]

    def _get(self, fn, shape):
        out = np.zeros(shape)
        self._ck(fn(self._h, _capi.ptr(out)))
        return out

    @property
    def population(self) -> np.ndarray:
        m = self.model
        return self._get(self._lib.mgr_get_populations, (m.ncells, m.linedata.nlev))

    @population.setter
    def population(self, pop: np.ndarray):
        pop = np.ascontiguousarray(pop, dtype=np.float64)
        self._ck(self._lib.mgr_set_populations(self._h, _capi.ptr(pop)))

    @property
    def J(self) -> np.ndarray:
        m = self.model
        return self._get(self._lib.mgr_get_J, (m.ncells, m.nfreqs))

    @property
    def Jlin(self) -> np.ndarray:
        m = self.model
        return self._get(self._lib.mgr_get_Jlin, (m.ncells, m.nlines))

    @property
    def Jeff(self) -> np.ndarray:
        m = self.model
        return self._get(self._lib.mgr_get_Jeff, (m.ncells, m.nlines))

    @property
    def Lambda(self) -> np.ndarray:
        """Diagonal ALO element Ls[p][k] (nr == p)."""
        m = self.model
        return self._get(self._lib.mgr_get_lambda, (m.ncells, m.nlines))

    @property
    def frequencies(self) -> np.ndarray:
        m = self.model
        return self._get(self._lib.mgr_get_frequencies, (m.ncells, m.nfreqs))

    def emissivity_opacity(self):
        m = self.model
        e = np.zeros((m.ncells, m.nlines))
        c = np.zeros((m.ncells, m.nlines))
        self._ck(self._lib.mgr_get_emissivity_opacity(self._h, _capi.ptr(e), _capi.ptr(c)))
        return e, c

    def convergence(self):
        f, r, x = C.c_double(), C.c_double(), C.c_double()
        self._ck(self._lib.mgr_get_convergence(self._h, C.byref(f), C.byref(r), C.byref(x)))
        return f.value, r.value, x.value

    def _record(self):
        f, r, x = self.convergence()
        self.fraction_not_converged.append(f)
        self.error_mean.append(r)
        self.error_max.append(x)

    def timer_start(self):
        self._ck(self._lib.mgr_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = C.c_double()
        self._ck(self._lib.mgr_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def launch_count(self) -> int:
        n = C.c_int64()
        self._ck(self._lib.mgr_get_launch_count(self._h, C.byref(n)))
        return n.value

    # ------------------------------------------------------ learned start
    def features(self) -> np.ndarray:
        out = np.zeros((self.model.ncells, _capi.MLP_FEATURES), np.float32)
        self._ck(self._lib.mgr_get_features(self._h, out.ctypes.data))
        return out

    def lte_logfrac(self) -> np.ndarray:
        out = np.zeros((self.model.ncells, self.model.linedata.nlev), np.float32)
        self._ck(self._lib.mgr_get_lte_logfrac(self._h, out.ctypes.data))
        return out

    def warm_start(self, net) -> int:
        """Learned start (replaces compute_LTE_level_populations)."""
        d = net.desc()
        return self._ck(self._lib.mgr_warm_start(self._h, C.byref(d)))

    def solve_trace_ms(self) -> float:
        """Of the last formal solve: ms spent rebuilding traces per batch of
        origins (0 when the traces are stored)."""
        t = C.c_double()
        self._ck(self._lib.mgr_get_solve_breakdown(self._h, C.byref(t)))
        return t.value

    def solve_stats(self):
        ms, up = C.c_double(), C.c_double()
        self._ck(self._lib.mgr_get_solve_stats(self._h, C.byref(ms), C.byref(up)))
        return ms.value, up.value
