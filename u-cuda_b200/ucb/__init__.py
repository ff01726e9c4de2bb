"""Python binding of the engine's C ABI (include/ucb.h) through ctypes.

The hot path runs in libucb.so (this directory): NVRTC-compiled sm_100a integrator
kernels driven by the C++ host code. There is no CPU fallback: every entry point fails
loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libucb.so"

UCB_OK, UCB_E_INVALID, UCB_E_COMPILE, UCB_E_CUDA, UCB_E_CANCELLED, UCB_E_NOGPU = range(6)
PREC_F64, PREC_F32 = 0, 1
PEAK_F32X2 = 2  # ucb_measure_fma_peak: packed FP32 pairs
MODE_NATIVE, MODE_EXACT = 0, 1
LLE_AUTO, LLE_SHADOW, LLE_TANGENT = 0, 1, 2


class UcbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[ucb error {code}] {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("mode", C.c_int32), ("lle_method", C.c_int32),
                ("nominal_steps", C.c_int32), ("block_threads", C.c_int32), ("max_registers", C.c_int32),
                ("unroll", C.c_int32), ("paired_cells", C.c_int32)]


class TuneReport(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("max_registers", C.c_int32), ("unroll", C.c_int32),
                ("candidates", C.c_int32), ("registers", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("best_ms", C.c_double), ("default_ms", C.c_double), ("wall_ms", C.c_double),
                ("trial_n_pts", C.c_int32), ("from_table", C.c_int32), ("key", C.c_char * 32),
                ("error", C.c_char * 256), ("confirm_default_ms", C.c_double), ("confirm_best_ms", C.c_double),
                ("confirm_n_pts", C.c_int32), ("pad0", C.c_int32)]

    def as_dict(self):
        return {f: (getattr(self, f).decode() if f in ("key", "error") else getattr(self, f))
                for f, _ in self._fields_}


class Lle2dRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32),
        ("sweep_over_var", C.c_int32), ("sweep_over_var_2", C.c_int32),
        ("sweep_over_h", C.c_int32), ("sweep_over_h_2", C.c_int32),
        ("log_scale", C.c_int32), ("log_scale_2", C.c_int32),
        ("param_index", C.c_int32), ("var_sweep_index", C.c_int32),
        ("param_index_2", C.c_int32), ("var_sweep_index_2", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("param_lo_2", C.c_double), ("param_hi_2", C.c_double),
        ("n_pts", C.c_int32),
        ("h", C.c_double), ("transient_time", C.c_double), ("t_max", C.c_double), ("NT", C.c_double),
        ("eps", C.c_double), ("max_value", C.c_double),
        ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)),
        ("opt", Options),
    ]


class Lle2dResult(C.Structure):
    _fields_ = [
        ("values", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("param_lo_2", C.c_double), ("param_hi_2", C.c_double),
        ("min_val", C.c_double), ("max_val", C.c_double), ("kernel_ms", C.c_double), ("steps", C.c_longlong),
        ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class Bif2dRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32),
        ("sweep_over_var", C.c_int32), ("sweep_over_var_2", C.c_int32),
        ("sweep_over_h", C.c_int32), ("sweep_over_h_2", C.c_int32),
        ("log_scale", C.c_int32), ("log_scale_2", C.c_int32),
        ("param_index", C.c_int32), ("var_sweep_index", C.c_int32),
        ("param_index_2", C.c_int32), ("var_sweep_index_2", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("param_lo_2", C.c_double), ("param_hi_2", C.c_double),
        ("n_pts", C.c_int32), ("writable_var", C.c_int32),
        ("h", C.c_double), ("transient_time", C.c_double), ("t_max", C.c_double), ("pre_scaller", C.c_int32),
        ("max_value", C.c_double), ("eps_dbscan", C.c_double), ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)), ("opt", Options),
    ]


class Bif2dResult(C.Structure):
    _fields_ = [
        ("values", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("param_lo_2", C.c_double), ("param_hi_2", C.c_double),
        ("min_val", C.c_double), ("max_val", C.c_double), ("kernel_ms", C.c_double), ("steps", C.c_longlong),
        ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class BasinsDbscanRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32), ("axis_x_var", C.c_int32), ("axis_y_var", C.c_int32),
        ("axis_x_lo", C.c_double), ("axis_x_hi", C.c_double), ("axis_y_lo", C.c_double), ("axis_y_hi", C.c_double),
        ("n_pts", C.c_int32), ("writable_var", C.c_int32),
        ("h", C.c_double), ("t_max", C.c_double), ("transient_time", C.c_double), ("pre_scaller", C.c_int32),
        ("max_value", C.c_double), ("eps_dbscan", C.c_double), ("feature1", C.c_int32), ("feature2", C.c_int32),
        ("mult1", C.c_double), ("mult2", C.c_double), ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)),
        ("progress_phase", C.POINTER(C.c_int32)), ("opt", Options),
    ]


class BasinsDbscanResult(C.Structure):
    _fields_ = [
        ("labels", C.POINTER(C.c_int32)), ("avg_peaks", C.POINTER(C.c_double)),
        ("avg_intervals", C.POINTER(C.c_double)), ("classes", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32),
        ("n_clusters", C.c_int32), ("min_cluster_idx", C.c_int32),
        ("avg_peaks_min", C.c_double), ("avg_peaks_max", C.c_double),
        ("avg_intervals_min", C.c_double), ("avg_intervals_max", C.c_double),
        ("kernel_ms", C.c_double), ("cluster_ms", C.c_double), ("steps", C.c_longlong),
        ("error", C.c_char * 1024),
    ]


class BasinsReclusterRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32), ("n_pts", C.c_int32), ("eps_dbscan", C.c_double),
        ("avg_peaks", C.POINTER(C.c_double)), ("avg_intervals", C.POINTER(C.c_double)),
        ("classes", C.POINTER(C.c_int32)), ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)),
        ("opt", Options),
    ]


class BasinsReclusterResult(C.Structure):
    _fields_ = [
        ("labels", C.POINTER(C.c_int32)), ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32),
        ("n_clusters", C.c_int32), ("min_cluster_idx", C.c_int32), ("cluster_ms", C.c_double),
        ("error", C.c_char * 1024),
    ]


class Lle1dRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32), ("sweep_over_var", C.c_int32), ("var_sweep_index", C.c_int32),
        ("sweep_over_h", C.c_int32), ("log_scale", C.c_int32), ("param_index", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("n_pts", C.c_int32),
        ("h", C.c_double), ("transient_time", C.c_double), ("t_max", C.c_double), ("NT", C.c_double),
        ("eps", C.c_double), ("max_value", C.c_double), ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)), ("opt", Options),
    ]


class Lle1dResult(C.Structure):
    _fields_ = [
        ("values", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("kernel_ms", C.c_double), ("steps", C.c_longlong),
        ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class Ls1dResult(C.Structure):
    _fields_ = [
        ("values", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32), ("n_exponents", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("kernel_ms", C.c_double), ("steps", C.c_longlong),
        ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class Bif1dRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32), ("param_index", C.c_int32), ("sweep_over_var", C.c_int32),
        ("var_sweep_index", C.c_int32), ("sweep_over_h", C.c_int32), ("log_scale", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("n_pts", C.c_int32), ("writable_var", C.c_int32),
        ("h", C.c_double), ("transient_time", C.c_double), ("t_max", C.c_double), ("pre_scaller", C.c_int32),
        ("max_value", C.c_double), ("max_peaks", C.c_int32), ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)), ("opt", Options),
    ]


class Bif1dResult(C.Structure):
    _fields_ = [
        ("counts", C.POINTER(C.c_int32)), ("peaks", C.POINTER(C.c_double)), ("intervals", C.POINTER(C.c_double)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32), ("record_steps", C.c_int32),
        ("param_lo", C.c_double), ("param_hi", C.c_double), ("kernel_ms", C.c_double), ("steps", C.c_longlong),
        ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class Ls2dRequest(C.Structure):
    _fields_ = Lle2dRequest._fields_ + [
        ("method", C.c_int32), ("gs_every", C.c_int32), ("rtol", C.c_double), ("atol", C.c_double),
        ("t_end", C.c_double), ("h0", C.c_double), ("max_steps", C.c_longlong),
    ]


class Ls2dResult(C.Structure):
    _fields_ = [
        ("values", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_int32)),
        ("min_val", C.POINTER(C.c_double)), ("max_val", C.POINTER(C.c_double)),
        ("cell_steps", C.POINTER(C.c_longlong)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32), ("n_exponents", C.c_int32),
        ("kernel_ms", C.c_double), ("steps", C.c_longlong), ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class BasinsRequest(C.Structure):
    _fields_ = [
        ("krs_body", C.c_char_p), ("amount_of_x", C.c_int32),
        ("initial_conditions", C.POINTER(C.c_double)), ("base_values", C.POINTER(C.c_double)),
        ("n_values", C.c_int32), ("axis_x_var", C.c_int32), ("axis_y_var", C.c_int32),
        ("axis_x_lo", C.c_double), ("axis_x_hi", C.c_double), ("axis_y_lo", C.c_double), ("axis_y_hi", C.c_double),
        ("n_pts", C.c_int32), ("period", C.c_double), ("steps_per_period", C.c_int32), ("max_periods", C.c_int32),
        ("match_count", C.c_int32), ("match_tol", C.c_double), ("phase_var", C.c_int32),
        ("max_value", C.c_double), ("merge_radius", C.c_double), ("csv_output_path", C.c_char_p),
        ("cancel", C.POINTER(C.c_int32)), ("progress", C.POINTER(C.c_float)), ("opt", Options),
    ]


MAX_ATTRACTORS = 256


class BasinsResult(C.Structure):
    _fields_ = [
        ("labels", C.POINTER(C.c_int32)), ("periods", C.POINTER(C.c_int32)), ("iterations", C.POINTER(C.c_int32)),
        ("ok", C.c_int32), ("cancelled", C.c_int32), ("n_pts", C.c_int32), ("n_attractors", C.c_int32),
        ("attractor_period", C.c_int32 * MAX_ATTRACTORS), ("attractor_point", (C.c_double * 2) * MAX_ATTRACTORS),
        ("kernel_ms", C.c_double), ("steps", C.c_longlong), ("flops", C.c_double), ("error", C.c_char * 1024),
    ]


class MlpConfig(C.Structure):
    _fields_ = [("fourier", C.c_int32), ("hidden", C.c_int32), ("layers", C.c_int32), ("fourier_scale", C.c_float),
                ("seed", C.c_uint64), ("batch", C.c_int32), ("train_steps", C.c_int32), ("lr", C.c_float),
                ("lr_final", C.c_float), ("beta_nll", C.c_float), ("reserved", C.c_int32 * 5)]


class SurrogateRequest(C.Structure):
    _fields_ = [("map", Lle2dRequest), ("train_pts", C.c_int32), ("sample_precision", C.c_int32),
                ("refine_precision", C.c_int32), ("pad0", C.c_int32), ("tol", C.c_double), ("coverage", C.c_double),
                ("sigma_max", C.c_double), ("lle_band", C.c_double), ("jump", C.c_double),
                ("min_predictable", C.c_double), ("mlp", MlpConfig)]


class SurrogateResult(C.Structure):
    _fields_ = [("ok", C.c_int32), ("n_pts", C.c_int32), ("n_samples", C.c_longlong), ("n_calib", C.c_longlong),
                ("n_refined", C.c_longlong), ("n_predicted", C.c_longlong), ("n_diverged", C.c_longlong),
                ("sigma_threshold", C.c_double), ("calib_within_tol", C.c_double),
                ("pilot_predictable", C.c_double), ("gated", C.c_int32), ("pad1", C.c_int32), ("sample_ms", C.c_double),
                ("train_ms", C.c_double), ("predict_ms", C.c_double), ("select_ms", C.c_double),
                ("refine_ms", C.c_double), ("total_ms", C.c_double), ("final_loss", C.c_float),
                ("pad0", C.c_float), ("error", C.c_char * 1024)]


LS_FIXED, LS_DP5 = 0, 1
_lib = None


def load():
    """Loads libucb.so (building it first if it is missing and nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("ucb_build", HERE.parent / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = C.CDLL(str(LIB_PATH))
    L.ucb_create.restype = C.c_void_p
    L.ucb_create.argtypes = [C.c_int]
    L.ucb_destroy.argtypes = [C.c_void_p]
    L.ucb_last_error.restype = C.c_char_p
    L.ucb_last_error.argtypes = [C.c_void_p]
    L.ucb_abi_version.restype = C.c_int
    L.ucb_kernel_launches.restype = C.c_longlong
    L.ucb_kernel_launches.argtypes = [C.c_void_p]
    L.ucb_clear_cache.argtypes = [C.c_void_p]
    L.ucb_default_options.argtypes = [C.POINTER(Options)]
    L.ucb_run_lle2d.restype = C.c_int
    L.ucb_run_lle2d.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest), C.POINTER(Lle2dResult)]
    L.ucb_lle2d_device.restype = C.c_int
    L.ucb_lle2d_device.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(Lle2dResult)]
    L.ucb_run_ls2d.restype = C.c_int
    L.ucb_run_ls2d.argtypes = [C.c_void_p, C.POINTER(Ls2dRequest), C.POINTER(Ls2dResult)]
    L.ucb_precompile_ls2d.restype = C.c_int
    L.ucb_precompile_ls2d.argtypes = [C.POINTER(Ls2dRequest), C.c_char_p, C.c_int]
    L.ucb_precompile_bif1d.restype = C.c_int
    L.ucb_precompile_bif1d.argtypes = [C.POINTER(Bif1dRequest), C.c_char_p, C.c_int]
    L.ucb_run_basins.restype = C.c_int
    L.ucb_run_basins.argtypes = [C.c_void_p, C.POINTER(BasinsRequest), C.POINTER(BasinsResult)]
    L.ucb_precompile_basins.restype = C.c_int
    L.ucb_precompile_basins.argtypes = [C.POINTER(BasinsRequest), C.c_char_p, C.c_int]
    L.ucb_run_bif1d.restype = C.c_int
    L.ucb_run_bif1d.argtypes = [C.c_void_p, C.POINTER(Bif1dRequest), C.POINTER(Bif1dResult)]
    L.ucb_prepare_lle2d.restype = C.c_int
    L.ucb_prepare_lle2d.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest)]
    L.ucb_lle2d_device_noalloc.restype = C.c_int
    L.ucb_lle2d_device_noalloc.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest), C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.POINTER(Lle2dResult)]
    L.ucb_lle2d_states.restype = C.c_int
    L.ucb_lle2d_states.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest), C.c_longlong, C.c_void_p]
    L.ucb_measure_fma_peak.restype = C.c_int
    L.ucb_measure_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.ucb_codegen.restype = C.c_int
    L.ucb_codegen.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_char_p, C.c_int,
                              C.c_char_p, C.c_int, C.c_char_p, C.c_int]
    L.ucb_precompile_lle2d.restype = C.c_int
    L.ucb_precompile_lle2d.argtypes = [C.POINTER(Lle2dRequest), C.c_char_p, C.c_int]
    L.ucb_run_bif2d.restype = C.c_int
    L.ucb_run_bif2d.argtypes = [C.c_void_p, C.POINTER(Bif2dRequest), C.POINTER(Bif2dResult)]
    L.ucb_precompile_bif2d.restype = C.c_int
    L.ucb_precompile_bif2d.argtypes = [C.POINTER(Bif2dRequest), C.c_char_p, C.c_int]
    L.ucb_run_basins_dbscan.restype = C.c_int
    L.ucb_run_basins_dbscan.argtypes = [C.c_void_p, C.POINTER(BasinsDbscanRequest), C.POINTER(BasinsDbscanResult)]
    L.ucb_precompile_basins_dbscan.restype = C.c_int
    L.ucb_precompile_basins_dbscan.argtypes = [C.POINTER(BasinsDbscanRequest), C.c_char_p, C.c_int]
    L.ucb_run_basins_recluster.restype = C.c_int
    L.ucb_run_basins_recluster.argtypes = [C.c_void_p, C.POINTER(BasinsReclusterRequest),
                                           C.POINTER(BasinsReclusterResult)]
    for fn, req in (("ucb_autotune_lle2d", Lle2dRequest), ("ucb_autotune_ls2d", Ls2dRequest),
                    ("ucb_autotune_basins", BasinsRequest), ("ucb_autotune_bif2d", Bif2dRequest)):
        getattr(L, fn).restype = C.c_int
        getattr(L, fn).argtypes = [C.c_void_p, C.POINTER(req), C.c_int32, C.POINTER(TuneReport)]
    L.ucb_run_lle1d.restype = C.c_int
    L.ucb_run_lle1d.argtypes = [C.c_void_p, C.POINTER(Lle1dRequest), C.POINTER(Lle1dResult)]
    L.ucb_run_ls1d.restype = C.c_int
    L.ucb_run_ls1d.argtypes = [C.c_void_p, C.POINTER(Lle1dRequest), C.POINTER(Ls1dResult)]
    L.ucb_lle2d_cells.restype = C.c_int
    L.ucb_lle2d_cells.argtypes = [C.c_void_p, C.POINTER(Lle2dRequest), C.c_void_p, C.c_longlong, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.POINTER(Lle2dResult)]
    L.ucb_mlp_default_config.argtypes = [C.POINTER(MlpConfig)]
    L.ucb_mlp_create.restype = C.c_void_p
    L.ucb_mlp_create.argtypes = [C.c_void_p, C.POINTER(MlpConfig)]
    L.ucb_mlp_destroy.argtypes = [C.c_void_p]
    L.ucb_mlp_param_count.restype = C.c_longlong
    L.ucb_mlp_param_count.argtypes = [C.c_void_p]
    for fn in ("ucb_mlp_get_params", "ucb_mlp_set_params", "ucb_mlp_get_fourier"):
        getattr(L, fn).restype = C.c_int
        getattr(L, fn).argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
    L.ucb_mlp_set_target_scale.restype = C.c_int
    L.ucb_mlp_set_target_scale.argtypes = [C.c_void_p, C.c_float, C.c_float]
    L.ucb_mlp_loss_grad.restype = C.c_int
    L.ucb_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.POINTER(C.c_float),
                                    C.c_void_p]
    L.ucb_mlp_fit.restype = C.c_int
    L.ucb_mlp_fit.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.POINTER(C.c_float)]
    L.ucb_mlp_predict.restype = C.c_int
    L.ucb_mlp_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ucb_default_surrogate_request.argtypes = [C.POINTER(SurrogateRequest)]
    L.ucb_run_lle2d_surrogate.restype = C.c_int
    L.ucb_run_lle2d_surrogate.argtypes = [C.c_void_p, C.POINTER(SurrogateRequest), C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.POINTER(SurrogateResult)]
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def options(precision=PREC_F64, mode=MODE_NATIVE, lle_method=LLE_AUTO, nominal_steps=False, block_threads=0,
            max_registers=0, unroll=0, paired_cells=False):
    """Run options; the launch-shape fields at 0 take the autotuned shape (or the default)."""
    o = Options()
    load().ucb_default_options(C.byref(o))
    o.precision, o.mode, o.lle_method = precision, mode, lle_method
    o.nominal_steps, o.block_threads = int(nominal_steps), block_threads
    o.max_registers, o.unroll, o.paired_cells = max_registers, unroll, int(paired_cells)
    return o


class Engine:
    """One engine object per device (the reference's ParametricEngine)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.h = self.lib.ucb_create(device)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ucb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(self.lib.ucb_kernel_launches(self.h))

    def last_error(self) -> str:
        return self.lib.ucb_last_error(self.h).decode()

    # ------------------------------------------------------------------ LLE 2D
    @staticmethod
    def lle2d_request(krs_body: str, amount_of_x: int, initial_conditions, base_values, *, n_pts,
                      param_index=0, param_index_2=0, var_sweep_index=0, var_sweep_index_2=0,
                      sweep_over_var=False, sweep_over_var_2=False, sweep_over_h=False, sweep_over_h_2=False,
                      log_scale=False, log_scale_2=False, param_lo=0.0, param_hi=1.0, param_lo_2=0.0,
                      param_hi_2=1.0, h=0.01, transient_time=0.0, t_max=100.0, NT=1.0, eps=1e-4,
                      max_value=1e6, csv_output_path=None, opt: Options | None = None):
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = Lle2dRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.sweep_over_var, r.sweep_over_var_2 = int(sweep_over_var), int(sweep_over_var_2)
        r.sweep_over_h, r.sweep_over_h_2 = int(sweep_over_h), int(sweep_over_h_2)
        r.log_scale, r.log_scale_2 = int(log_scale), int(log_scale_2)
        r.param_index, r.var_sweep_index = param_index, var_sweep_index
        r.param_index_2, r.var_sweep_index_2 = param_index_2, var_sweep_index_2
        r.param_lo, r.param_hi, r.param_lo_2, r.param_hi_2 = param_lo, param_hi, param_lo_2, param_hi_2
        r.n_pts = n_pts
        r.h, r.transient_time, r.t_max, r.NT, r.eps, r.max_value = h, transient_time, t_max, NT, eps, max_value
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_lle2d(self, req: Lle2dRequest, values=None, flags=None):
        n = req.n_pts
        if values is None:
            values = np.empty(max(n, 0) ** 2, dtype=np.float64)
        if flags is None:
            flags = np.empty(max(n, 0) ** 2, dtype=np.int32)
        res = Lle2dResult()
        res.values = _dptr(values)
        res.flags = flags.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_lle2d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return values, flags, res

    # ------------------------------------------------------------------ bifurcation 2D
    @staticmethod
    def bif2d_request(krs_body: str, amount_of_x: int, initial_conditions, base_values, *, n_pts,
                      param_index=0, param_index_2=0, var_sweep_index=0, var_sweep_index_2=0,
                      sweep_over_var=False, sweep_over_var_2=False, sweep_over_h=False, sweep_over_h_2=False,
                      log_scale=False, log_scale_2=False, param_lo=0.0, param_hi=1.0, param_lo_2=0.0,
                      param_hi_2=1.0, writable_var=0, h=0.01, transient_time=0.0, t_max=100.0, pre_scaller=1,
                      max_value=1e6, eps_dbscan=0.1, csv_output_path=None, opt: Options | None = None):
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = Bif2dRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.sweep_over_var, r.sweep_over_var_2 = int(sweep_over_var), int(sweep_over_var_2)
        r.sweep_over_h, r.sweep_over_h_2 = int(sweep_over_h), int(sweep_over_h_2)
        r.log_scale, r.log_scale_2 = int(log_scale), int(log_scale_2)
        r.param_index, r.var_sweep_index = param_index, var_sweep_index
        r.param_index_2, r.var_sweep_index_2 = param_index_2, var_sweep_index_2
        r.param_lo, r.param_hi, r.param_lo_2, r.param_hi_2 = param_lo, param_hi, param_lo_2, param_hi_2
        r.n_pts, r.writable_var = n_pts, writable_var
        r.h, r.transient_time, r.t_max, r.pre_scaller = h, transient_time, t_max, pre_scaller
        r.max_value, r.eps_dbscan = max_value, eps_dbscan
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_bif2d(self, req: Bif2dRequest):
        n = req.n_pts
        values = np.empty(max(n, 0) ** 2, dtype=np.float64)
        flags = np.empty(max(n, 0) ** 2, dtype=np.int32)
        res = Bif2dResult()
        res.values = _dptr(values)
        res.flags = flags.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_bif2d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return values, flags, res

    # ------------------------------------------------------------------ LLE / LS 1D
    @staticmethod
    def lle1d_request(krs_body: str, amount_of_x: int, initial_conditions, base_values, *, n_pts, param_index=0,
                      sweep_over_var=False, var_sweep_index=0, sweep_over_h=False, log_scale=False, param_lo=0.0,
                      param_hi=1.0, h=0.01, transient_time=0.0, t_max=100.0, NT=1.0, eps=1e-4, max_value=1e6,
                      csv_output_path=None, opt: Options | None = None):
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = Lle1dRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.sweep_over_var, r.var_sweep_index = int(sweep_over_var), var_sweep_index
        r.sweep_over_h, r.log_scale, r.param_index = int(sweep_over_h), int(log_scale), param_index
        r.param_lo, r.param_hi, r.n_pts = param_lo, param_hi, n_pts
        r.h, r.transient_time, r.t_max, r.NT, r.eps, r.max_value = h, transient_time, t_max, NT, eps, max_value
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_lle1d(self, req: Lle1dRequest):
        n = req.n_pts
        values = np.empty(max(n, 0), dtype=np.float64)
        flags = np.empty(max(n, 0), dtype=np.int32)
        res = Lle1dResult()
        res.values = _dptr(values)
        res.flags = flags.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_lle1d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return values, flags, res

    def run_ls1d(self, req: Lle1dRequest):
        n, nx = req.n_pts, req.amount_of_x
        values = np.empty(max(n, 0) * nx, dtype=np.float64)
        flags = np.empty(max(n, 0), dtype=np.int32)
        res = Ls1dResult()
        res.values = _dptr(values)
        res.flags = flags.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_ls1d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return values.reshape(n, nx), flags, res

    # ------------------------------------------------------------------ LS 2D
    @staticmethod
    def ls2d_request(krs_body, amount_of_x, initial_conditions, base_values, *, method=0, gs_every=10, rtol=0.0,
                     atol=0.0, t_end=0.0, h0=0.0, max_steps=0, **kw):
        base = Engine.lle2d_request(krs_body, amount_of_x, initial_conditions, base_values, **kw)
        r = Ls2dRequest()
        for name, _ in Lle2dRequest._fields_:
            setattr(r, name, getattr(base, name))
        r._keep = base._keep
        r.method, r.gs_every, r.rtol, r.atol, r.t_end, r.h0, r.max_steps = method, gs_every, rtol, atol, t_end, h0, \
            max_steps
        return r

    def run_ls2d(self, req: Ls2dRequest, cell_steps=False):
        """-> (values[k, cell], flags, result); with cell_steps=True result.cell_work holds the
        per-cell steps (fixed) / step attempts (DP5)."""
        n, nx = req.n_pts, req.amount_of_x
        values = np.empty(max(n, 0) ** 2 * nx, dtype=np.float64)
        flags = np.empty(max(n, 0) ** 2, dtype=np.int32)
        mn = np.empty(nx, dtype=np.float64)
        mx = np.empty(nx, dtype=np.float64)
        res = Ls2dResult()
        res.values = _dptr(values)
        res.flags = flags.ctypes.data_as(C.POINTER(C.c_int32))
        res.min_val = _dptr(mn)
        res.max_val = _dptr(mx)
        work = np.zeros(max(n, 0) ** 2, dtype=np.int64) if cell_steps else None
        if cell_steps:
            res.cell_steps = work.ctypes.data_as(C.POINTER(C.c_longlong))
        rc = self.lib.ucb_run_ls2d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        res.cell_work = work
        return values.reshape(nx, n * n), flags, res

    # ------------------------------------------------------------------ basins
    @staticmethod
    def basins_request(krs_body, amount_of_x, initial_conditions, base_values, *, n_pts, axis_x_var=0,
                       axis_y_var=1, axis_x_lo=-1.0, axis_x_hi=1.0, axis_y_lo=-1.0, axis_y_hi=1.0, period=1.0,
                       steps_per_period=100, max_periods=2000, match_count=20, match_tol=1e-6, phase_var=-1,
                       max_value=1e6, merge_radius=0.0, csv_output_path=None, opt: Options | None = None):
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = BasinsRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.axis_x_var, r.axis_y_var = axis_x_var, axis_y_var
        r.axis_x_lo, r.axis_x_hi, r.axis_y_lo, r.axis_y_hi = axis_x_lo, axis_x_hi, axis_y_lo, axis_y_hi
        r.n_pts, r.period, r.steps_per_period, r.max_periods = n_pts, period, steps_per_period, max_periods
        r.match_count, r.match_tol, r.phase_var = match_count, match_tol, phase_var
        r.max_value, r.merge_radius = max_value, merge_radius
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_basins(self, req: BasinsRequest):
        n = req.n_pts
        labels = np.empty(n * n, dtype=np.int32)
        periods = np.empty(n * n, dtype=np.int32)
        iters = np.empty(n * n, dtype=np.int32)
        res = BasinsResult()
        res.labels = labels.ctypes.data_as(C.POINTER(C.c_int32))
        res.periods = periods.ctypes.data_as(C.POINTER(C.c_int32))
        res.iterations = iters.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_basins(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        att = [(res.attractor_period[i], res.attractor_point[i][0], res.attractor_point[i][1])
               for i in range(min(res.n_attractors, MAX_ATTRACTORS))]
        return labels, periods, iters, att, res

    # ------------------------------------------------------------------ basins (reference method)
    @staticmethod
    def basins_dbscan_request(krs_body, amount_of_x, initial_conditions, base_values, *, n_pts, axis_x_var=0,
                              axis_y_var=1, axis_x_lo=-10.0, axis_x_hi=10.0, axis_y_lo=-10.0, axis_y_hi=10.0,
                              writable_var=0, h=0.01, t_max=1000.0, transient_time=10000.0, pre_scaller=1,
                              max_value=1e6, eps_dbscan=0.5, feature1=0, feature2=1, mult1=1.0, mult2=1.0,
                              csv_output_path=None, opt: Options | None = None):
        """Request of run_basins (BasinsRequest, parametric_engine.h:659-691), its defaults."""
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = BasinsDbscanRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.axis_x_var, r.axis_y_var = axis_x_var, axis_y_var
        r.axis_x_lo, r.axis_x_hi, r.axis_y_lo, r.axis_y_hi = axis_x_lo, axis_x_hi, axis_y_lo, axis_y_hi
        r.n_pts, r.writable_var = n_pts, writable_var
        r.h, r.t_max, r.transient_time, r.pre_scaller = h, t_max, transient_time, pre_scaller
        r.max_value, r.eps_dbscan = max_value, eps_dbscan
        r.feature1, r.feature2, r.mult1, r.mult2 = feature1, feature2, mult1, mult2
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_basins_dbscan(self, req: BasinsDbscanRequest):
        """-> (labels, avg_peaks, avg_intervals, classes, result), row-major iy*n + ix."""
        n = req.n_pts
        labels = np.empty(max(n, 0) ** 2, dtype=np.int32)
        f1 = np.empty(max(n, 0) ** 2, dtype=np.float64)
        f2 = np.empty(max(n, 0) ** 2, dtype=np.float64)
        cls = np.empty(max(n, 0) ** 2, dtype=np.int32)
        res = BasinsDbscanResult()
        res.labels = labels.ctypes.data_as(C.POINTER(C.c_int32))
        res.avg_peaks = _dptr(f1)
        res.avg_intervals = _dptr(f2)
        res.classes = cls.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_basins_dbscan(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return labels, f1, f2, cls, res

    def run_basins_recluster(self, krs_body, amount_of_x, n_pts, eps_dbscan, avg_peaks, avg_intervals, classes,
                             opt: Options | None = None):
        """DBSCAN of given features (run_basins_recluster) -> (labels, result)."""
        f1 = np.ascontiguousarray(avg_peaks, dtype=np.float64)
        f2 = np.ascontiguousarray(avg_intervals, dtype=np.float64)
        cls = np.ascontiguousarray(classes, dtype=np.int32)
        if not (len(f1) == len(f2) == len(cls) == n_pts * n_pts):
            raise UcbError(UCB_E_INVALID, "features / classes: size does not match n_pts^2")
        req = BasinsReclusterRequest()
        body = krs_body.encode()
        req.krs_body, req.amount_of_x, req.n_pts, req.eps_dbscan = body, amount_of_x, n_pts, eps_dbscan
        req.avg_peaks, req.avg_intervals = _dptr(f1), _dptr(f2)
        req.classes = cls.ctypes.data_as(C.POINTER(C.c_int32))
        req.opt = opt if opt is not None else options()
        labels = np.empty(n_pts * n_pts, dtype=np.int32)
        res = BasinsReclusterResult()
        res.labels = labels.ctypes.data_as(C.POINTER(C.c_int32))
        rc = self.lib.ucb_run_basins_recluster(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return labels, res

    # ------------------------------------------------------------------ autotuning
    def autotune(self, req, force=False) -> dict:
        """Launch-shape search for the kernel `req` would run (ucb_autotune_*); later runs
        with the shape fields of their options at 0 use the result."""
        fn = {Lle2dRequest: "ucb_autotune_lle2d", Ls2dRequest: "ucb_autotune_ls2d",
              BasinsRequest: "ucb_autotune_basins", Bif2dRequest: "ucb_autotune_bif2d"}[type(req)]
        rep = TuneReport()
        rc = getattr(self.lib, fn)(self.h, C.byref(req), int(force), C.byref(rep))
        if rc != UCB_OK:
            raise UcbError(rc, rep.error.decode() or self.last_error())
        return rep.as_dict()

    # ------------------------------------------------------------------ bifurcation 1D
    @staticmethod
    def bif1d_request(krs_body: str, amount_of_x: int, initial_conditions, base_values, *, n_pts, param_index=0,
                      sweep_over_var=False, var_sweep_index=0, sweep_over_h=False, log_scale=False, param_lo=0.0,
                      param_hi=1.0, writable_var=0, h=0.01, transient_time=0.0, t_max=100.0, pre_scaller=1,
                      max_value=1e6, max_peaks=64, csv_output_path=None, opt: Options | None = None):
        ic = np.ascontiguousarray(initial_conditions, dtype=np.float64)
        vals = np.ascontiguousarray(base_values, dtype=np.float64)
        r = Bif1dRequest()
        r._keep = (ic, vals, krs_body.encode())
        r.krs_body = r._keep[2]
        r.amount_of_x = amount_of_x
        r.initial_conditions = _dptr(ic)
        r.base_values = _dptr(vals)
        r.n_values = len(vals)
        r.param_index, r.sweep_over_var, r.var_sweep_index = param_index, int(sweep_over_var), var_sweep_index
        r.sweep_over_h, r.log_scale = int(sweep_over_h), int(log_scale)
        r.param_lo, r.param_hi, r.n_pts, r.writable_var = param_lo, param_hi, n_pts, writable_var
        r.h, r.transient_time, r.t_max, r.pre_scaller = h, transient_time, t_max, pre_scaller
        r.max_value, r.max_peaks = max_value, max_peaks
        r.csv_output_path = csv_output_path.encode() if csv_output_path else None
        r.opt = opt if opt is not None else options()
        return r

    def run_bif1d(self, req: Bif1dRequest):
        n, mp = req.n_pts, max(req.max_peaks, 0)
        counts = np.empty(max(n, 0), dtype=np.int32)
        peaks = np.empty(max(n, 0) * mp, dtype=np.float64)
        intervals = np.empty(max(n, 0) * mp, dtype=np.float64)
        res = Bif1dResult()
        res.counts = counts.ctypes.data_as(C.POINTER(C.c_int32))
        res.peaks = _dptr(peaks)
        res.intervals = _dptr(intervals)
        rc = self.lib.ucb_run_bif1d(self.h, C.byref(req), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return counts, peaks.reshape(n, mp), intervals.reshape(n, mp), res

    def prepare_lle2d(self, req: Lle2dRequest):
        """One-time set-up for lle2d_device_noalloc (compiles/loads the kernel, finds the
        scratch array's device address)."""
        rc = self.lib.ucb_prepare_lle2d(self.h, C.byref(req))
        if rc != UCB_OK:
            raise UcbError(rc, self.last_error())

    def lle2d_device_noalloc(self, req: Lle2dRequest, d_values_ptr: int, d_flags_ptr: int, stream_ptr: int = 0):
        """LLE map into caller-owned device buffers with no device allocation (scratch in a
        fixed array of the library; n_pts <= 4096; calls overlapping on the GPU race)."""
        res = Lle2dResult()
        rc = self.lib.ucb_lle2d_device_noalloc(self.h, C.byref(req), C.c_void_p(d_values_ptr),
                                               C.c_void_p(d_flags_ptr), C.c_void_p(stream_ptr), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return res

    def lle2d_states(self, req: Lle2dRequest, n_steps: int):
        n = req.n_pts
        out = np.empty(n * n * req.amount_of_x, dtype=np.float64)
        rc = self.lib.ucb_lle2d_states(self.h, C.byref(req), n_steps, out.ctypes.data_as(C.c_void_p))
        if rc != UCB_OK:
            raise UcbError(rc, self.last_error())
        return out.reshape(n * n, req.amount_of_x)

    def lle2d_device(self, req: Lle2dRequest, d_values_ptr: int, d_flags_ptr: int, stream_ptr: int = 0):
        res = Lle2dResult()
        rc = self.lib.ucb_lle2d_device(self.h, C.byref(req), C.c_void_p(d_values_ptr), C.c_void_p(d_flags_ptr),
                                       C.c_void_p(stream_ptr), C.byref(res))
        if rc != UCB_OK:
            raise UcbError(rc, res.error.decode())
        return res


def mlp_config(**kw) -> MlpConfig:
    c = MlpConfig()
    load().ucb_mlp_default_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Mlp:
    """The BF16 tensor-core MLP of the surrogate (ucb_mlp_* entry points)."""

    def __init__(self, engine: Engine, cfg: MlpConfig | None = None, **kw):
        self.engine = engine
        self.lib = engine.lib
        self.cfg = cfg if cfg is not None else mlp_config(**kw)
        self.h = self.lib.ucb_mlp_create(engine.h, C.byref(self.cfg))
        if not self.h:
            raise UcbError(UCB_E_INVALID, engine.last_error())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ucb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != UCB_OK:
            raise UcbError(rc, self.engine.last_error())

    @property
    def n_params(self) -> int:
        return int(self.lib.ucb_mlp_param_count(self.h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(self.lib.ucb_mlp_get_params(self.h, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.lib.ucb_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p), p.size))

    def fourier(self) -> np.ndarray:
        out = np.empty((self.cfg.fourier, 2), dtype=np.float32)
        self._check(self.lib.ucb_mlp_get_fourier(self.h, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    def set_target_scale(self, mean: float, std: float):
        self._check(self.lib.ucb_mlp_set_target_scale(self.h, mean, std))

    def loss_grad(self, u, y):
        u = np.ascontiguousarray(u, dtype=np.float32).reshape(-1, 2)
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_float(0)
        self._check(self.lib.ucb_mlp_loss_grad(self.h, u.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                               len(y), C.byref(loss), g.ctypes.data_as(C.c_void_p)))
        return float(loss.value), g

    def fit(self, d_u_ptr: int, d_y_ptr: int, n: int, stream_ptr: int = 0) -> float:
        loss = C.c_float(0)
        self._check(self.lib.ucb_mlp_fit(self.h, C.c_void_p(d_u_ptr), C.c_void_p(d_y_ptr), n,
                                         C.c_void_p(stream_ptr), C.byref(loss)))
        return float(loss.value)

    def predict(self, d_u_ptr: int, n: int, d_mean_ptr: int, d_std_ptr: int, stream_ptr: int = 0):
        self._check(self.lib.ucb_mlp_predict(self.h, C.c_void_p(d_u_ptr), n, C.c_void_p(d_mean_ptr),
                                             C.c_void_p(d_std_ptr), C.c_void_p(stream_ptr)))


def surrogate_request(map_req: Lle2dRequest, **kw) -> SurrogateRequest:
    """Surrogate-refined map request around an LLE-2D request (defaults from the library;
    keyword `mlp` takes a dict of MlpConfig fields)."""
    r = SurrogateRequest()
    load().ucb_default_surrogate_request(C.byref(r))
    r.map = map_req
    r._keep = map_req._keep
    mlp = kw.pop("mlp", None)
    for k, v in kw.items():
        setattr(r, k, v)
    if mlp:
        for k, v in mlp.items():
            setattr(r.mlp, k, v)
    return r


def _engine_surrogate(self, req: SurrogateRequest, d_values_ptr: int, d_flags_ptr: int, stream_ptr: int = 0):
    res = SurrogateResult()
    rc = self.lib.ucb_run_lle2d_surrogate(self.h, C.byref(req), C.c_void_p(d_values_ptr), C.c_void_p(d_flags_ptr),
                                          C.c_void_p(stream_ptr), C.byref(res))
    if rc != UCB_OK:
        raise UcbError(rc, res.error.decode())
    return res


def _engine_cells(self, req: Lle2dRequest, d_cells_ptr: int, n_cells: int, d_values_ptr: int, d_flags_ptr: int,
                  stream_ptr: int = 0):
    res = Lle2dResult()
    rc = self.lib.ucb_lle2d_cells(self.h, C.byref(req), C.c_void_p(d_cells_ptr), n_cells, C.c_void_p(d_values_ptr),
                                  C.c_void_p(d_flags_ptr), C.c_void_p(stream_ptr), C.byref(res))
    if rc != UCB_OK:
        raise UcbError(rc, res.error.decode())
    return res


Engine.run_lle2d_surrogate = _engine_surrogate
Engine.lle2d_cells = _engine_cells


def precompile_lle2d(req) -> str:
    """Compiles the sm_100a kernel a run with this request would use (no GPU needed)."""
    fn = {Lle2dRequest: "ucb_precompile_lle2d", Ls2dRequest: "ucb_precompile_ls2d",
          Bif1dRequest: "ucb_precompile_bif1d", BasinsRequest: "ucb_precompile_basins",
          Bif2dRequest: "ucb_precompile_bif2d",
          BasinsDbscanRequest: "ucb_precompile_basins_dbscan"}[type(req)]
    buf = C.create_string_buffer(65536)
    rc = getattr(load(), fn)(C.byref(req), buf, len(buf))
    if rc != UCB_OK:
        raise UcbError(rc, buf.value.decode(errors="replace"))
    return buf.value.decode(errors="replace")


def measure_fma_peak(precision=PREC_F64) -> float:
    """FMA-pipe throughput of the current device in TFLOP/s (roofline denominator)."""
    v = C.c_double(0)
    rc = load().ucb_measure_fma_peak(precision, C.byref(v))
    if rc != UCB_OK:
        raise UcbError(rc, "fma probe failed")
    return v.value


SCHEMES = {"Euler": 0, "Euler-Cromer": 1, "Explicit Midpoint": 2, "RK4": 3, "DOPRI78": 4, "CD": 5}


def codegen(text: str, alphabet: str, scheme: str = "RK4", order_as_in_system=False, func_defs: str | None = None):
    """System text -> (step body, variables, parameters)."""
    out = C.create_string_buffer(1 << 20)
    vs = C.create_string_buffer(4096)
    ps = C.create_string_buffer(4096)
    rc = load().ucb_codegen(text.encode(), alphabet.encode(), int(order_as_in_system),
                            func_defs.encode() if func_defs else None, SCHEMES[scheme], out, len(out), vs, len(vs),
                            ps, len(ps))
    if rc != UCB_OK:
        raise UcbError(rc, out.value.decode())
    split = lambda b: [x for x in b.value.decode().split(",") if x]
    return out.value.decode(), split(vs), split(ps)


precompile = precompile_lle2d
