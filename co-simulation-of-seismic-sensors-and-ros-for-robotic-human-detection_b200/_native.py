"""ctypes binding of libgfk (include/gfk.h).

There is no fallback: if libgfk.so is missing or cannot be loaded, importing
the engine raises, and if no CUDA device is present, opening a context raises.
"""
import ctypes
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libgfk.so"

# status codes (enum gfk_status)
OK, EARG, ESTACK, EGUARD, ESINGULAR, ENONFINITE, ETIMEOUT, ECUDA, ENOMEM, EIO, ELIMIT = range(11)
STATUS_NAMES = {OK: "OK", EARG: "EARG", ESTACK: "ESTACK", EGUARD: "EGUARD", ESINGULAR: "ESINGULAR",
                ENONFINITE: "ENONFINITE", ETIMEOUT: "ETIMEOUT", ECUDA: "ECUDA", ENOMEM: "ENOMEM", EIO: "EIO",
                ELIMIT: "ELIMIT"}

REFERENCE_DIRECT = 0
DUNKIN = 1
PLAIN_FP64 = 0
SPLIT_INT8 = 1
LOSS_PLAIN = 0
LOSS_COMPLEX = 1
LOSS_AMPLITUDE = 2
NET_TIMES = 6
NET_FOURIER = 47

# every symbol include/gfk.h declares
EXPORTS = [
    "gfk_open", "gfk_close", "gfk_status_string", "gfk_last_error", "gfk_kernel_launches", "gfk_stream", "gfk_selftest_wait_timeout",
    "gfk_stack_validate", "gfk_check_layer_phase", "gfk_grid_for",
    "gfk_surface_response", "gfk_static_coefficient", "gfk_vertical_displacement",
    "gfk_vertical_displacement_multi", "gfk_bank_spectra", "gfk_bank_payload",
    "gfk_plan_create", "gfk_plan_execute", "gfk_plan_result_device", "gfk_plan_download",
    "gfk_plan_execute_download",
    "gfk_plan_launches_per_execute", "gfk_plan_tuning", "gfk_prop_shape", "gfk_plan_quad_shape", "gfk_plan_kernel_times", "gfk_plan_destroy",
    "gfk_plan_use_graph", "gfk_batch_create",
    "gfk_bank_pack", "gfk_bank_write", "gfk_vertical_displacement_multi_noalloc",
    "gfk_dispersion_modes", "gfk_secular", "gfk_fdtd_grid", "gfk_fdtd_run",
    "gfk_trace_metrics", "gfk_ensemble_gate", "gfk_scatter_rows", "gfk_bank_tables", "gfk_bank_impulse_responses",
    "gfk_bank_device_open", "gfk_bank_device_impulse_responses", "gfk_bank_device_close",
    "gfk_dataset_create", "gfk_dataset_fill", "gfk_dataset_stats", "gfk_dataset_labels", "gfk_dataset_destroy",
    "gfk_net_create", "gfk_net_set_scales", "gfk_net_train", "gfk_net_train_ranges", "gfk_net_predict", "gfk_net_evaluate",
    "gfk_net_param_count", "gfk_net_params", "gfk_net_fourier", "gfk_net_probe", "gfk_net_destroy",
]


class GfkLayer(ctypes.Structure):
    _fields_ = [("thickness_m", ctypes.c_double), ("vp_mps", ctypes.c_double), ("vs_mps", ctypes.c_double),
                ("density_kgm3", ctypes.c_double), ("qs", ctypes.c_double), ("qp", ctypes.c_double)]


class GfkMedium(ctypes.Structure):
    _fields_ = [("layers", ctypes.POINTER(GfkLayer)), ("count", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("ref_freq_hz", ctypes.c_double), ("default_q", ctypes.c_double),
                ("sls_tau_sigma", ctypes.c_double), ("sls_tau_eps", ctypes.c_double)]


class GfkIntegration(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int32), ("_pad", ctypes.c_int32), ("kmax_factor", ctypes.c_double),
                ("kmax", ctypes.c_double)]


class GfkGrid(ctypes.Structure):
    _fields_ = [("kmax", ctypes.c_double), ("samples", ctypes.c_int32), ("_pad", ctypes.c_int32)]


class GfkSolve(ctypes.Structure):
    _fields_ = [("formulation", ctypes.c_int32), ("quadrature", ctypes.c_int32), ("guard", ctypes.c_int32),
                ("_pad", ctypes.c_int32), ("omega_imag", ctypes.c_double)]


class GfkFdtdModel(ctypes.Structure):
    _fields_ = [("medium", GfkMedium), ("max_range_m", ctypes.c_double), ("depth_m", ctypes.c_double),
                ("spacing_m", ctypes.c_double), ("pml_cells", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("pml_reflection", ctypes.c_double), ("dominant_freq_hz", ctypes.c_double),
                ("courant", ctypes.c_double)]


class GfkSearch(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int32), ("_pad", ctypes.c_int32), ("tolerance", ctypes.c_double)]


class GfkNetConfig(ctypes.Structure):
    _fields_ = [("nsoil_scalars", ctypes.c_int32), ("batch", ctypes.c_int32), ("warmup_steps", ctypes.c_int32),
                ("total_steps", ctypes.c_int32), ("lr_max", ctypes.c_float), ("lr_min", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("weight_decay", ctypes.c_float), ("phase_weight", ctypes.c_float),
                ("fourier_sigma", ctypes.c_float), ("loss_mode", ctypes.c_int32), ("weight_floor", ctypes.c_float),
                ("phase_cap", ctypes.c_float), ("_pad", ctypes.c_int32), ("seed", ctypes.c_uint64)]


_lib = None


def lib():
    """The loaded libgfk; raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"libgfk is not built ({LIB_PATH} missing); run build.build() — "
                           "there is no CPU fallback")
    L = ctypes.CDLL(str(LIB_PATH))
    P, d, i32, i64, f32 = ctypes.POINTER, ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    vp = ctypes.c_void_p
    sig = {
        "gfk_open": (ctypes.c_int, [ctypes.c_int, P(vp)]),
        "gfk_close": (ctypes.c_int, [vp]),
        "gfk_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "gfk_last_error": (ctypes.c_char_p, [vp]),
        "gfk_kernel_launches": (i64, [vp]),
        "gfk_stream": (vp, [vp]),
        "gfk_selftest_wait_timeout": (ctypes.c_int, [vp, i64, P(i32)]),
        "gfk_stack_validate": (ctypes.c_int, [P(GfkMedium)]),
        "gfk_check_layer_phase": (ctypes.c_int, [P(GfkMedium), d]),
        "gfk_grid_for": (ctypes.c_int, [P(GfkMedium), P(d), i32, d, GfkIntegration, P(GfkGrid)]),
        "gfk_surface_response": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), P(d), P(d), i64, P(d)]),
        "gfk_static_coefficient": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), d, d, P(d)]),
        "gfk_vertical_displacement": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), d, d, GfkIntegration, P(d)]),
        "gfk_vertical_displacement_multi": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), P(d), i32, d,
                                                           GfkIntegration, P(d)]),
        "gfk_bank_spectra": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), P(d), i32, P(d), i32, GfkIntegration,
                                            P(d), P(i32)]),
        "gfk_bank_payload": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), P(d), i32, P(d), i32, GfkIntegration, i32,
                                            i32, P(ctypes.c_float), P(i32)]),
        "gfk_plan_create": (ctypes.c_int, [vp, P(GfkMedium), P(GfkSolve), P(d), i32, P(d), i32, GfkIntegration,
                                           P(vp)]),
        "gfk_plan_execute": (ctypes.c_int, [vp]),
        "gfk_plan_result_device": (ctypes.c_int, [vp, P(vp)]),
        "gfk_plan_download": (ctypes.c_int, [vp, P(d), P(i32)]),
        "gfk_plan_execute_download": (ctypes.c_int, [vp, P(d), P(i32)]),
        "gfk_plan_launches_per_execute": (i32, [vp]),
        "gfk_plan_tuning": (ctypes.c_int, [vp, P(i32), P(ctypes.c_float), i32]),
        "gfk_plan_quad_shape": (ctypes.c_int, [vp, P(i32), P(i32), P(ctypes.c_float), i32]),
        "gfk_prop_shape": (ctypes.c_int, [i32, P(i32), P(i32), P(i32), P(i32), P(i32)]),
        "gfk_plan_kernel_times": (ctypes.c_int, [vp, P(d), P(d), P(d), i32]),
        "gfk_plan_destroy": (ctypes.c_int, [vp]),
        "gfk_plan_use_graph": (ctypes.c_int, [vp, i32]),
        "gfk_batch_create": (ctypes.c_int, [vp, P(GfkMedium), i32, P(P(d)), P(i32), P(GfkSolve), P(d), i32,
                                            GfkIntegration, P(vp)]),
        "gfk_bank_pack": (ctypes.c_int, [P(d), i32, i32, i32, i32, P(ctypes.c_float)]),
        "gfk_bank_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, P(ctypes.c_float), i64]),
        "gfk_vertical_displacement_multi_noalloc": (ctypes.c_int, [P(GfkMedium), P(GfkSolve), P(d), i32, d,
                                                                   GfkIntegration, P(d), vp]),
        "gfk_fdtd_grid": (ctypes.c_int, [P(GfkFdtdModel), P(d), P(i32), P(i32)]),
        "gfk_fdtd_run": (ctypes.c_int, [vp, P(GfkFdtdModel), P(d), i32, P(d), i32, i32, P(d), P(d), P(d)]),
        "gfk_dispersion_modes": (ctypes.c_int, [vp, P(GfkMedium), P(d), i32, GfkSearch, i32, P(d), P(i32)]),
        "gfk_secular": (ctypes.c_int, [vp, P(GfkMedium), P(d), P(d), i64, P(d), P(i32)]),
        "gfk_ensemble_gate": (ctypes.c_int, [vp, P(vp), i32, i64, i32, i32, P(d), d, d, vp, P(ctypes.c_uint8),
                                             P(d)]),
        "gfk_scatter_rows": (ctypes.c_int, [vp, vp, i64, P(i64), i64, vp]),
        "gfk_bank_tables": (ctypes.c_int, [vp, P(f32), i32, i32, P(d), P(d)]),
        "gfk_bank_impulse_responses": (ctypes.c_int, [vp, P(f32), i32, i32, d, d, d, i32, P(d), i32, P(d), i32, i32,
                                                      P(d)]),
        "gfk_bank_device_open": (ctypes.c_int, [vp, P(f32), i32, i32, d, d, d, i32, P(vp)]),
        "gfk_bank_device_impulse_responses": (ctypes.c_int, [vp, P(d), i32, P(d), i32, i32, vp, i32]),
        "gfk_bank_device_close": (ctypes.c_int, [vp]),
        "gfk_trace_metrics": (ctypes.c_int, [vp, vp, i64, i32, i32, P(d), i32, d, d, i32, i32, P(d), P(d)]),
        "gfk_dataset_create": (ctypes.c_int, [vp, i32, i32, P(d), P(d), P(d), i32, P(d), i32, d, P(vp)]),
        "gfk_dataset_fill": (ctypes.c_int, [vp, vp, i32, i32]),
        "gfk_dataset_stats": (ctypes.c_int, [vp, P(d)]),
        "gfk_dataset_labels": (ctypes.c_int, [vp, i32, P(f32)]),
        "gfk_dataset_destroy": (ctypes.c_int, [vp]),
        "gfk_net_create": (ctypes.c_int, [vp, P(GfkNetConfig), P(vp)]),
        "gfk_net_set_scales": (ctypes.c_int, [vp, d, d, d, d, P(f32)]),
        "gfk_net_train": (ctypes.c_int, [vp, vp, P(i32), i32, i32, P(f32)]),
        "gfk_net_train_ranges": (ctypes.c_int, [vp, vp, P(i32), i32, i32, i32, i32, P(f32)]),
        "gfk_net_predict": (ctypes.c_int, [vp, P(d), P(d), i32, P(d), i32, P(d), i32, vp, i32]),
        "gfk_net_evaluate": (ctypes.c_int, [vp, vp, P(i32), i32, P(d)]),
        "gfk_net_param_count": (i64, [vp]),
        "gfk_net_params": (ctypes.c_int, [vp, P(f32), i64, i32]),
        "gfk_net_fourier": (ctypes.c_int, [vp, P(f32), i32]),
        "gfk_net_probe": (ctypes.c_int, [vp, P(f32), P(f32), P(f32), P(f32), P(f32)]),
        "gfk_net_destroy": (ctypes.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def status_string(code):
    return lib().gfk_status_string(code).decode()
