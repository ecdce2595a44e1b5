"""ctypes front-end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the plain-C restatement of Magritte's radiation hot path in
``oracle/magritte_oracle.c``.  It is the checker the CUDA path is compared
against and the CPU baseline timed beside it; the product package never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmagritte_oracle.so")
_lib = None

_P = C.c_void_p
_i64 = C.c_int64
_dbl = C.c_double


class _Colpar(C.Structure):
    _fields_ = [("ntmp", C.c_int32), ("ncol", C.c_int32), ("ortho_para", C.c_int32),
                ("pad_", C.c_int32), ("icol", _P), ("jcol", _P), ("tmp", _P), ("Cd", _P),
                ("Ce", _P), ("abundance", _P)]


class _Model(C.Structure):
    _fields_ = [("ncells", _i64), ("position", _P), ("velocity", _P), ("nbr_offsets", _P),
                ("nbr_list", _P), ("boundary", _P), ("cell2boundary", _P), ("nboundary", _i64),
                ("boundary2cell", _P), ("boundary_temperature", _P), ("nrays", _i64),
                ("rays", _P), ("ray_weights", _P), ("temperature", _P), ("vturb2", _P),
                ("nlev", C.c_int32), ("nrad", C.c_int32), ("energy", _P), ("weight", _P),
                ("irad", _P), ("jrad", _P), ("A", _P), ("Bs", _P), ("Ba", _P),
                ("frequency", _P), ("inverse_mass", _dbl), ("population_tot", _P),
                ("nquads", C.c_int32), ("ncolpar", C.c_int32), ("quad_roots", _P),
                ("quad_weights", _P), ("colpar", _P), ("pop_prec", _dbl),
                ("max_width_fraction", _dbl)]


class _State(C.Structure):
    _fields_ = [("nfreqs", _i64), ("nu", _P), ("nr_line", _P), ("corr_k", _P), ("corr_z", _P),
                ("appears", _P), ("I_bdy", _P), ("pop", _P), ("prev1", _P), ("prev2", _P),
                ("prev3", _P), ("emissivity", _P), ("opacity", _P), ("J", _P), ("Ls", _P),
                ("Jlin", _P), ("Jeff", _P), ("Jdif", _P), ("fnc", _dbl), ("rcm", _dbl),
                ("max_rel", _dbl), ("trace_errors", _i64), ("lu_errors", _i64),
                ("n_off_diag", _i64), ("Loff", _P), ("Loff_nr", _P)]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    src = os.path.join(_HERE, "magritte_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "ORACLE_CC=gcc"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_const.restype = _dbl
        L.orc_const.argtypes = [C.c_int]
        L.orc_dshift_max.restype = _dbl
        L.orc_dshift_max.argtypes = [_P, _i64]
        L.orc_doppler_shift.restype = _dbl
        L.orc_doppler_shift.argtypes = [_P, _i64, _i64, _i64, C.c_int, _P]
        L.orc_npoints_on_ray.restype = _i64
        L.orc_npoints_on_ray.argtypes = [_P, _i64, _i64, _dbl, _P]
        L.orc_trace_ray.restype = _i64
        L.orc_trace_ray.argtypes = [_P, _i64, _i64, _dbl, _i64, _P, _P, _P, _P]
        for n in ("orc_spectral_discretisation", "orc_boundary_intensities",
                  "orc_statistical_equilibrium"):
            getattr(L, n).restype = C.c_int
            getattr(L, n).argtypes = [_P, _P]
        for n in ("orc_lte", "orc_set_emissivity_opacity", "orc_compute_jeff",
                  "orc_check_convergence", "orc_ng_acceleration"):
            getattr(L, n).restype = None
            getattr(L, n).argtypes = [_P, _P]
        L.orc_compute_radiation_field.restype = C.c_int
        L.orc_compute_radiation_field.argtypes = [_P, _P, _P, _P, _i64, _i64, C.c_int]
        L.orc_solve_raypair.restype = None
        L.orc_solve_raypair.argtypes = [_i64, _i64, _P, _P, _dbl, _dbl, _P, _P]
        L.orc_compute_radiation_field_scattering.restype = C.c_int
        L.orc_compute_radiation_field_scattering.argtypes = [_P, _P, _P, _P, _P, _P, _P, C.c_int]
        L.orc_calc_U_and_V.restype = None
        L.orc_calc_U_and_V.argtypes = [_P, _P, _P, _P, _P, _P]
        L.orc_image_discretisation.restype = C.c_int
        L.orc_image_discretisation.argtypes = [_P, _P, _dbl]
        L.orc_compute_image.restype = C.c_int
        L.orc_compute_image.argtypes = [_P, _P, _P, _i64, _P, _P, C.c_int]
        L.orc_raypair_lambda_row.restype = None
        L.orc_raypair_lambda_row.argtypes = [_i64, _i64, _P, _P, _i64, _P, _P, _P]
        L.orc_compute_level_populations.restype = _i64
        L.orc_compute_level_populations.argtypes = [_P, _P, _P, C.c_int, _i64, _dbl, C.c_int, _P]
        L.orc_compute_level_populations_ng.restype = _i64
        L.orc_compute_level_populations_ng.argtypes = [_P, _P, _P, C.c_int, _i64, _dbl, C.c_int,
                                                       _P, C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def solve_raypair(n_ar: int, term1: np.ndarray, dtau: np.ndarray, I0: float, In: float):
    """u and the diagonal ALO element at the origin of one ray pair, by the
    reference's elimination + back substitution (raypair_solver.tpp:200-334)."""
    term1 = np.ascontiguousarray(term1, dtype=np.float64)
    dtau = np.ascontiguousarray(dtau, dtype=np.float64)
    u = np.zeros(1)
    L = np.zeros(1)
    lib().orc_solve_raypair(n_ar, term1.shape[0], _ptr(term1), _ptr(dtau), I0, In, _ptr(u), _ptr(L))
    return float(u[0]), float(L[0])


def raypair_lambda_row(n_ar: int, term1: np.ndarray, dtau: np.ndarray, n_off_diag: int):
    """The origin's row of one ray pair's Lambda operator from the non-local
    branch of RayPair::solve: (diagonal, [n_off_diag-1] elements toward the
    front, [n_off_diag-1] toward the back)."""
    term1 = np.ascontiguousarray(term1, dtype=np.float64)
    dtau = np.ascontiguousarray(dtau, dtype=np.float64)
    n = max(1, n_off_diag - 1)
    diag, lo, up = np.zeros(1), np.zeros(n), np.zeros(n)
    lib().orc_raypair_lambda_row(n_ar, term1.shape[0], _ptr(term1), _ptr(dtau), n_off_diag,
                                 _ptr(diag), _ptr(lo), _ptr(up))
    return float(diag[0]), lo[:n_off_diag - 1], up[:n_off_diag - 1]


class Oracle:
    """Holds a model and the oracle's state arrays, mirroring the order of
    calls a Magritte user makes (``tests/integration/test_0_1D_all_constant.py:64-99``)."""

    def __init__(self, model):
        self.m = model
        L = lib()
        N, nl, nr = model.ncells, model.linedata.nlev, model.nlines
        nf = model.nfreqs
        ld = model.linedata
        keep = self._keep = []

        def k(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a

        self.antipod = k(model.antipod(), np.int64)
        bmask = k(model.boundary_mask(), np.uint8)
        c2b = np.full(N, N, dtype=np.int64)
        c2b[model.boundary2cell] = np.arange(model.nboundary)
        c2b = k(c2b, np.int64)
        self.cell2boundary = c2b
        cps = (_Colpar * max(1, len(ld.colpar)))()
        for i, cp in enumerate(ld.colpar):
            abn = k(model.abundance[:, cp.num_col_partner], np.float64)
            cps[i].ntmp = cp.tmp.shape[0]
            cps[i].ncol = cp.icol.shape[0]
            cps[i].ortho_para = {"n": 0, "o": 1, "p": 2}[cp.orth_or_para_H2]
            cps[i].icol = _ptr(k(cp.icol, np.int64))
            cps[i].jcol = _ptr(k(cp.jcol, np.int64))
            cps[i].tmp = _ptr(k(cp.tmp, np.float64))
            cps[i].Cd = _ptr(k(cp.Cd, np.float64))
            cps[i].Ce = _ptr(k(cp.Ce, np.float64))
            cps[i].abundance = _ptr(abn)
        keep.append(cps)
        mm = _Model()
        mm.ncells = N
        mm.position = _ptr(k(model.position, np.float64))
        mm.velocity = _ptr(k(model.velocity, np.float64))
        mm.nbr_offsets = _ptr(k(model.nbr_offsets, np.int64))
        mm.nbr_list = _ptr(k(model.nbr_list, np.int64))
        mm.boundary = _ptr(bmask)
        mm.cell2boundary = _ptr(c2b)
        mm.nboundary = model.nboundary
        mm.boundary2cell = _ptr(k(model.boundary2cell, np.int64))
        mm.boundary_temperature = _ptr(k(model.boundary_temperature, np.float64))
        mm.nrays = model.nrays
        mm.rays = _ptr(k(model.rays, np.float64))
        mm.ray_weights = _ptr(k(model.ray_weights, np.float64))
        mm.temperature = _ptr(k(model.temperature, np.float64))
        mm.vturb2 = _ptr(k(model.vturb2, np.float64))
        mm.nlev = nl
        mm.nrad = nr
        mm.energy = _ptr(k(ld.energy, np.float64))
        mm.weight = _ptr(k(ld.weight, np.float64))
        mm.irad = _ptr(k(ld.irad, np.int64))
        mm.jrad = _ptr(k(ld.jrad, np.int64))
        mm.A = _ptr(k(ld.A, np.float64))
        mm.Bs = _ptr(k(ld.Bs, np.float64))
        mm.Ba = _ptr(k(ld.Ba, np.float64))
        mm.frequency = _ptr(k(ld.frequency, np.float64))
        mm.inverse_mass = ld.inverse_mass
        mm.population_tot = _ptr(k(model.population_tot, np.float64))
        mm.nquads = model.nquads
        mm.ncolpar = len(ld.colpar)
        mm.quad_roots = _ptr(k(model.quad_roots, np.float64))
        mm.quad_weights = _ptr(k(model.quad_weights, np.float64))
        mm.colpar = C.addressof(cps)
        mm.pop_prec = model.pop_prec
        mm.max_width_fraction = model.max_width_fraction
        self._model = mm

        z = lambda *shape, dt=np.float64: np.zeros(shape, dtype=dt)
        self.nu = z(N, nf)
        self.nr_line = z(N, nr, model.nquads, dt=np.int64)
        self.corr_k = z(nf, dt=np.int64)
        self.corr_z = z(nf, dt=np.int64)
        self.appears = z(nf, dt=np.uint8)
        self.I_bdy = z(model.nboundary, nf)
        self.pop = z(N, nl)
        self.prev1 = z(N, nl)
        self.prev2 = z(N, nl)
        self.prev3 = z(N, nl)
        self.emissivity = z(N, nr)
        self.opacity = z(N, nr)
        self.J = z(N, nf)
        self.Ls = z(N, nr)
        self.Jlin = z(N, nr)
        self.Jeff = z(N, nr)
        self.Jdif = z(N, nr)
        st = _State()
        st.nfreqs = nf
        for name in ("nu", "nr_line", "corr_k", "corr_z", "appears", "I_bdy", "pop", "prev1",
                     "prev2", "prev3", "emissivity", "opacity", "J", "Ls", "Jlin", "Jeff", "Jdif"):
            setattr(st, name, _ptr(getattr(self, name)))
        self._state = st
        self.M = C.byref(self._model)
        self.S = C.byref(self._state)
        self.identity_sort = None

    # --------------------------------------------------------------- set-up
    def compute_spectral_discretisation(self) -> int:
        bad = lib().orc_spectral_discretisation(self.M, self.S)
        self.identity_sort = (bad == 0)
        return 0

    def compute_boundary_intensities(self) -> int:
        return lib().orc_boundary_intensities(self.M, self.S)

    def compute_LTE_level_populations(self) -> int:
        lib().orc_lte(self.M, self.S)
        lib().orc_set_emissivity_opacity(self.M, self.S)
        return 0

    def set_n_off_diag(self, n_off_diag: int):
        """parameters.n_off_diag: with M >= 2 the formal solve also keeps the
        M-1 nearest off-diagonal ALO elements on each side of every ray pair
        (``Loff`` [N, nrad, npairs, 2, M-1] and their cells ``Loff_nr``
        [N, npairs, 2, M-1], -1 where the pair has no such point), and the
        statistical equilibrium solves the rate equations of all cells as one
        system."""
        m = self.m
        M1 = max(0, int(n_off_diag) - 1)
        np_ = m.nrays // 2
        self.Loff = np.zeros((m.ncells, m.nlines, np_, 2, max(M1, 1)))
        self.Loff_nr = np.full((m.ncells, np_, 2, max(M1, 1)), -1, dtype=np.int64)
        self._state.n_off_diag = int(n_off_diag)
        self._state.Loff = _ptr(self.Loff)
        self._state.Loff_nr = _ptr(self.Loff_nr)
        return self

    def setup(self):
        self.compute_spectral_discretisation()
        self.compute_boundary_intensities()
        self.compute_LTE_level_populations()
        return self

    def set_populations(self, pop: np.ndarray):
        self.pop[...] = pop
        lib().orc_set_emissivity_opacity(self.M, self.S)

    # ---------------------------------------------------------- scattering
    def compute_radiation_field_scattering(self, U, V, nthreads: int = 0):
        """Every ray pair and origin through setup_using_scattering and
        solve_using_scattering with scattering terms U, V
        [nrays/2, ncells, nfreqs]; returns u, v at the origins (same shape).
        J and the ALO are accumulated as in compute_radiation_field."""
        m = self.m
        shape = (m.nrays // 2, m.ncells, m.nfreqs)
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(shape)
        V = np.ascontiguousarray(V, dtype=np.float64).reshape(shape)
        u = np.zeros(shape)
        v = np.zeros(shape)
        err = lib().orc_compute_radiation_field_scattering(self.M, self.S, _ptr(self.antipod),
                                                           _ptr(U), _ptr(V), _ptr(u), _ptr(v),
                                                           nthreads)
        if err:
            raise RuntimeError("trace error")
        return u, v

    def calc_U_and_V(self, u, v):
        m = self.m
        shape = (m.nrays // 2, m.ncells, m.nfreqs)
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(shape)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(shape)
        U = np.zeros(shape)
        V = np.zeros(shape)
        lib().orc_calc_U_and_V(self.M, self.S, _ptr(u), _ptr(v), _ptr(U), _ptr(V))
        return U, V

    # -------------------------------------------------------------- images
    def compute_spectral_discretisation_image(self, width: float) -> int:
        """The same grid line + line*width*root (sorted) in every cell
        (sim_spectrum.tpp:200-250); the boundary table follows the grid."""
        lib().orc_image_discretisation(self.M, self.S, float(width))
        return lib().orc_boundary_intensities(self.M, self.S)

    def compute_image(self, r: int, nthreads: int = 0):
        """(I_m, I_p) [ncells, nfreqs] of compute_and_write_image for ray r
        (sim_radiation.tpp:348-478)."""
        m = self.m
        I_m = np.zeros((m.ncells, m.nfreqs))
        I_p = np.zeros((m.ncells, m.nfreqs))
        err = lib().orc_compute_image(self.M, self.S, _ptr(self.antipod), int(r), _ptr(I_m),
                                      _ptr(I_p), nthreads)
        if err:
            raise RuntimeError("trace error while imaging")
        return I_m, I_p

    # ------------------------------------------------------------ geometry
    def dshift_max(self, o: int) -> float:
        return lib().orc_dshift_max(self.M, o)

    def doppler_shift(self, origin: int, ray: int, current: int, rest: bool = False) -> float:
        return lib().orc_doppler_shift(self.M, origin, ray, current, int(rest), _ptr(self.antipod))

    def npoints_on_ray(self, o: int, r: int) -> int:
        err = np.zeros(1, dtype=np.int64)
        n = lib().orc_npoints_on_ray(self.M, o, r, self.dshift_max(o), _ptr(err))
        if err[0]:
            raise RuntimeError(f"trace error {int(err[0])} at origin {o} ray {r}")
        return int(n)

    def trace_ray(self, o: int, r: int):
        cap = self.npoints_on_ray(o, r)
        cell = np.zeros(max(cap, 1), dtype=np.int64)
        shift = np.zeros(max(cap, 1))
        dZ = np.zeros(max(cap, 1))
        err = np.zeros(1, dtype=np.int64)
        n = lib().orc_trace_ray(self.M, o, r, self.dshift_max(o), cap, _ptr(cell), _ptr(shift),
                                _ptr(dZ), _ptr(err))
        if err[0]:
            raise RuntimeError(f"trace error {int(err[0])} at origin {o} ray {r}")
        return cell[:n], shift[:n], dZ[:n]

    def get_npoints_on_rays(self) -> np.ndarray:
        """npoints[r][o] = n_ar + n_r + 1 (simulation.tpp:540-552)."""
        m = self.m
        out = np.zeros((m.nrays // 2, m.ncells), dtype=np.int64)
        for r in range(m.nrays // 2):
            ar = int(self.antipod[r])
            for o in range(m.ncells):
                out[r, o] = self.npoints_on_ray(o, r) + self.npoints_on_ray(o, ar) + 1
        return out

    # ----------------------------------------------------------- transfer
    def compute_radiation_field(self, origins=None, npairs: int = 0, nthreads: int = 0) -> int:
        if origins is None:
            return lib().orc_compute_radiation_field(self.M, self.S, _ptr(self.antipod), None, 0,
                                                     npairs, nthreads)
        o = np.ascontiguousarray(origins, dtype=np.int64)
        return lib().orc_compute_radiation_field(self.M, self.S, _ptr(self.antipod), _ptr(o),
                                                 o.shape[0], npairs, nthreads)

    def compute_Jeff(self):
        lib().orc_compute_jeff(self.M, self.S)

    def compute_level_populations_from_stateq(self) -> int:
        err = lib().orc_statistical_equilibrium(self.M, self.S)
        lib().orc_check_convergence(self.M, self.S)
        lib().orc_set_emissivity_opacity(self.M, self.S)
        return err

    def ng_acceleration(self):
        lib().orc_ng_acceleration(self.M, self.S)
        lib().orc_check_convergence(self.M, self.S)
        lib().orc_set_emissivity_opacity(self.M, self.S)

    def compute_level_populations(self, use_ng: bool = True, max_iter: int = 1000,
                                  tol_max_rel: float = 0.0, nthreads: int = 0,
                                  ng_every: int = 4):
        hist = np.zeros(max_iter)
        it = lib().orc_compute_level_populations_ng(self.M, self.S, _ptr(self.antipod),
                                                    int(use_ng), max_iter, tol_max_rel, nthreads,
                                                    _ptr(hist), int(ng_every))
        return int(it), hist[:it].copy()

    @property
    def fraction_not_converged(self) -> float:
        return self._state.fnc

    @property
    def relative_change_mean(self) -> float:
        return self._state.rcm

    @property
    def relative_change_max(self) -> float:
        return self._state.max_rel

    @property
    def trace_errors(self) -> int:
        return self._state.trace_errors

    @property
    def lu_errors(self) -> int:
        return self._state.lu_errors
