"""ctypes binding of the C ABI in ``include/magritte_b200.h``.

The shared library is built in-tree (``magritte_b200/libmagritte_b200.so``).
There is no fallback: if the library is missing or cannot be loaded, every
call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MAGRITTE_B200_LIB") or os.path.join(HERE, "libmagritte_b200.so")

MGR_OK = 0
STATUS_NAMES = {
    0: "MGR_OK", 1: "MGR_ERR_INVALID_ARG", 2: "MGR_ERR_TRACE", 3: "MGR_ERR_LU_SINGULAR",
    4: "MGR_ERR_NOT_CONVERGED", 5: "MGR_ERR_CUDA", 6: "MGR_ERR_TIMEOUT",
    7: "MGR_ERR_UNSUPPORTED", 8: "MGR_ERR_STATE", 9: "MGR_ERR_NO_MEMORY",
    10: "MGR_ERR_TOO_LARGE",
}
MGR_FP64 = 0
MGR_MIXED = 1

# Every function the header declares (checked by the CPU test suite).
EXPORTS = (
    "mgr_create", "mgr_destroy", "mgr_last_error", "mgr_version", "mgr_upload_model",
    "mgr_set_trace_budget", "mgr_compute_spectral_discretisation",
    "mgr_compute_boundary_intensities", "mgr_compute_LTE_level_populations", "mgr_trace",
    "mgr_get_npoints_on_rays", "mgr_get_trace", "mgr_compute_radiation_field", "mgr_set_keep_J",
    "mgr_compute_Jeff", "mgr_compute_level_populations_from_stateq", "mgr_ng_acceleration",
    "mgr_get_convergence", "mgr_compute_level_populations", "mgr_set_populations",
    "mgr_get_populations", "mgr_get_J", "mgr_get_Jlin", "mgr_get_Jeff", "mgr_get_lambda",
    "mgr_get_emissivity_opacity", "mgr_get_frequencies", "mgr_get_solve_stats",
    "mgr_synchronize", "mgr_timer_start", "mgr_timer_stop", "mgr_get_launch_count",
    "mgr_convergence_noalloc", "mgr_mlp_param_count", "mgr_get_features", "mgr_get_lte_logfrac",
    "mgr_warm_start", "mgr_mlp_train", "mgr_mlp_forward", "mgr_mlp_loss_grad",
    "mgr_set_segments", "mgr_get_segment_results", "mgr_set_autotune", "mgr_get_tuning",
    "mgr_get_patch_stats", "mgr_set_origin_range", "mgr_stateq_local", "mgr_stateq_finish",
    "mgr_get_device_buffer", "mgr_get_population_history", "mgr_set_population_history",
    "mgr_compute_image", "mgr_set_patch_capacity", "mgr_set_scattering_terms",
    "mgr_get_scattering_terms", "mgr_compute_radiation_field_scattering", "mgr_get_scattering_uv",
    "mgr_calc_U_and_V", "mgr_get_solve_breakdown", "mgr_set_n_off_diag", "mgr_get_alo_nonlocal",
    "mgr_get_nonlocal_sweeps",
)
# mgr_buffer
BUF_POPULATION, BUF_PREV1, BUF_PREV2, BUF_PREV3, BUF_JLIN, BUF_LAMBDA, BUF_PARTIALS = range(7)
CELLS_PER_PARTIAL = 4
MLP_FEATURES = 10
MLP_HIDDEN = 128
NOALLOC_MAX_ELEMENTS = 67108864

_P = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32
_dbl = C.c_double


class ColparDesc(C.Structure):
    _fields_ = [("ntmp", _i32), ("ncol", _i32), ("ortho_para", _i32), ("reserved", _i32),
                ("icol", _P), ("jcol", _P), ("tmp", _P), ("Cd", _P), ("Ce", _P),
                ("abundance", _P)]


class ModelDesc(C.Structure):
    _fields_ = [("ncells", _i64), ("position", _P), ("velocity", _P), ("nbr_offsets", _P),
                ("nbr_list", _P), ("nboundary", _i64), ("boundary2cell", _P),
                ("boundary_temperature", _P), ("nrays", _i64), ("rays", _P),
                ("ray_weights", _P), ("temperature", _P), ("vturb2", _P), ("nlev", _i32),
                ("nrad", _i32), ("energy", _P), ("weight", _P), ("irad", _P), ("jrad", _P),
                ("A", _P), ("Bs", _P), ("Ba", _P), ("frequency", _P), ("inverse_mass", _dbl),
                ("population_tot", _P), ("nquads", _i32), ("ncolpar", _i32),
                ("quad_roots", _P), ("quad_weights", _P), ("colpar", _P), ("pop_prec", _dbl),
                ("max_width_fraction", _dbl)]


class MlpDesc(C.Structure):
    _fields_ = [("nin", _i32), ("nout", _i32), ("params", _P), ("feat_mean", _P),
                ("feat_istd", _P)]


class TrainOpts(C.Structure):
    _fields_ = [("epochs", _i32), ("batch", _i32), ("lr", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_uint64)]


class AliOpts(C.Structure):
    _fields_ = [("use_ng", _i32), ("precision", _i32), ("max_iter", _i64),
                ("tol_max_rel", _dbl), ("use_graph", _i32), ("ng_every", _i32)]


class Tuning(C.Structure):
    _fields_ = [("kernel", _i32), ("min_blocks", _i32), ("warps_per_block", _i32),
                ("tuned", _i32), ("ms", C.c_float * 8)]


class MagritteError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(build_if_missing: bool = True):
    """Loads the CUDA library (building it first when absent or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and LIB_PATH == os.path.join(HERE, "libmagritte_b200.so"):
        from . import build as _build
        if _build.stale():
            _build.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH}")
    L = C.CDLL(LIB_PATH)
    for name in EXPORTS:
        getattr(L, name).restype = C.c_int
    L.mgr_last_error.restype = C.c_char_p
    L.mgr_last_error.argtypes = [_P]
    L.mgr_version.restype = C.c_char_p
    L.mgr_version.argtypes = []
    L.mgr_create.argtypes = [C.c_int, C.POINTER(_P)]
    L.mgr_destroy.argtypes = [_P]
    L.mgr_upload_model.argtypes = [_P, C.POINTER(ModelDesc)]
    L.mgr_set_trace_budget.argtypes = [_P, _i64]
    for n in ("mgr_compute_spectral_discretisation", "mgr_compute_boundary_intensities",
              "mgr_compute_LTE_level_populations", "mgr_trace", "mgr_compute_Jeff",
              "mgr_compute_level_populations_from_stateq", "mgr_ng_acceleration",
              "mgr_synchronize", "mgr_timer_start"):
        getattr(L, n).argtypes = [_P]
    L.mgr_timer_stop.argtypes = [_P, C.POINTER(_dbl)]
    L.mgr_get_launch_count.argtypes = [_P, C.POINTER(_i64)]
    L.mgr_get_npoints_on_rays.argtypes = [_P, _P]
    L.mgr_get_trace.argtypes = [_P, _i64, _i64, _i64, _P, _P, _P, C.POINTER(_i64)]
    L.mgr_compute_radiation_field.argtypes = [_P, _i32]
    L.mgr_set_keep_J.argtypes = [_P, _i32]
    L.mgr_get_convergence.argtypes = [_P, C.POINTER(_dbl), C.POINTER(_dbl), C.POINTER(_dbl)]
    L.mgr_compute_level_populations.argtypes = [_P, C.POINTER(AliOpts), C.POINTER(_i64), _P]
    for n in ("mgr_set_populations", "mgr_get_populations", "mgr_get_J", "mgr_get_Jlin",
              "mgr_get_Jeff", "mgr_get_lambda", "mgr_get_frequencies"):
        getattr(L, n).argtypes = [_P, _P]
    L.mgr_get_emissivity_opacity.argtypes = [_P, _P, _P]
    L.mgr_get_solve_stats.argtypes = [_P, C.POINTER(_dbl), C.POINTER(_dbl)]
    L.mgr_convergence_noalloc.argtypes = [_P, _P, _P, _i64, _i32, _dbl, _P, _P]
    L.mgr_set_origin_range.argtypes = [_P, _i64, _i64]
    L.mgr_stateq_local.argtypes = [_P]
    L.mgr_stateq_finish.argtypes = [_P]
    L.mgr_get_device_buffer.argtypes = [_P, _i32, C.POINTER(_P), C.POINTER(_i64)]
    L.mgr_get_population_history.argtypes = [_P, _P, _P, _P]
    L.mgr_compute_image.argtypes = [_P, _i64, _dbl, _P, _P, _P, _P, _P]
    L.mgr_set_patch_capacity.argtypes = [_P, _i64]
    L.mgr_set_n_off_diag.argtypes = [_P, C.c_int32]
    L.mgr_get_alo_nonlocal.argtypes = [_P, _P, _P]
    L.mgr_get_nonlocal_sweeps.argtypes = [_P, _P]
    L.mgr_set_scattering_terms.argtypes = [_P, _P, _P]
    L.mgr_get_scattering_terms.argtypes = [_P, _P, _P]
    L.mgr_compute_radiation_field_scattering.argtypes = [_P]
    L.mgr_get_scattering_uv.argtypes = [_P, _P, _P]
    L.mgr_calc_U_and_V.argtypes = [_P]
    L.mgr_get_solve_breakdown.argtypes = [_P, C.POINTER(_dbl)]
    L.mgr_set_population_history.argtypes = [_P, _P, _P, _P, _P]
    L.mgr_mlp_param_count.argtypes = [_i32, C.POINTER(_i64)]
    L.mgr_get_features.argtypes = [_P, _P]
    L.mgr_get_lte_logfrac.argtypes = [_P, _P]
    L.mgr_warm_start.argtypes = [_P, C.POINTER(MlpDesc)]
    L.mgr_mlp_train.argtypes = [C.c_int, C.POINTER(MlpDesc), _P, _P, _P, _i64, C.POINTER(TrainOpts), _P]
    L.mgr_mlp_forward.argtypes = [C.c_int, C.POINTER(MlpDesc), _P, _i64, _P]
    L.mgr_mlp_loss_grad.argtypes = [C.c_int, C.POINTER(MlpDesc), _P, _P, _P, _i64, _P, _P]
    L.mgr_set_segments.argtypes = [_P, _i64, _P]
    L.mgr_get_patch_stats.argtypes = [_P, C.POINTER(_i64), C.POINTER(_i64)]
    L.mgr_get_segment_results.argtypes = [_P, _P, _P]
    L.mgr_set_autotune.argtypes = [_P, _i32]
    L.mgr_get_tuning.argtypes = [_P, _i32, C.POINTER(Tuning)]
    _lib = L
    return L


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def make_desc(model):
    """Builds the ModelDesc of a :class:`magritte_b200.model.Model`; returns
    the descriptor and the list of arrays it points into (keep it alive)."""
    keep = []

    def k(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return ptr(a)

    ld = model.linedata
    cps = (ColparDesc * max(1, len(ld.colpar)))()
    for i, cp in enumerate(ld.colpar):
        cps[i].ntmp = cp.tmp.shape[0]
        cps[i].ncol = cp.icol.shape[0]
        cps[i].ortho_para = {"n": 0, "o": 1, "p": 2}[cp.orth_or_para_H2]
        cps[i].icol = k(cp.icol, np.int64)
        cps[i].jcol = k(cp.jcol, np.int64)
        cps[i].tmp = k(cp.tmp, np.float64)
        cps[i].Cd = k(cp.Cd, np.float64)
        cps[i].Ce = k(cp.Ce, np.float64)
        cps[i].abundance = k(model.abundance[:, cp.num_col_partner], np.float64)
    keep.append(cps)
    d = ModelDesc()
    d.ncells = model.ncells
    d.position = k(model.position, np.float64)
    d.velocity = k(model.velocity, np.float64)
    d.nbr_offsets = k(model.nbr_offsets, np.int64)
    d.nbr_list = k(model.nbr_list, np.int64)
    d.nboundary = model.nboundary
    d.boundary2cell = k(model.boundary2cell, np.int64)
    d.boundary_temperature = k(model.boundary_temperature, np.float64)
    d.nrays = model.nrays
    d.rays = k(model.rays, np.float64)
    d.ray_weights = k(model.ray_weights, np.float64)
    d.temperature = k(model.temperature, np.float64)
    d.vturb2 = k(model.vturb2, np.float64)
    d.nlev = ld.nlev
    d.nrad = ld.nrad
    d.energy = k(ld.energy, np.float64)
    d.weight = k(ld.weight, np.float64)
    d.irad = k(ld.irad, np.int64)
    d.jrad = k(ld.jrad, np.int64)
    d.A = k(ld.A, np.float64)
    d.Bs = k(ld.Bs, np.float64)
    d.Ba = k(ld.Ba, np.float64)
    d.frequency = k(ld.frequency, np.float64)
    d.inverse_mass = ld.inverse_mass
    d.population_tot = k(model.population_tot, np.float64)
    d.nquads = model.nquads
    d.ncolpar = len(ld.colpar)
    d.quad_roots = k(model.quad_roots, np.float64)
    d.quad_weights = k(model.quad_weights, np.float64)
    d.colpar = C.addressof(cps)
    d.pop_prec = model.pop_prec
    d.max_width_fraction = model.max_width_fraction
    return d, keep
