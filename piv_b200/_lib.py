"""ctypes binding of libpivb200.so (declarations mirror include/piv_b200.h).

The library is built in-tree (piv_b200/libpivb200.so). There is no fallback: if it is missing or
fails to load, every entry point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpivb200.so")

PIV_OK, PIV_ERR_CONFIG, PIV_ERR_SHAPE_MISMATCH, PIV_ERR_IMAGE_TOO_SMALL = 0, 1, 2, 3
PIV_ERR_FRAME_RATE, PIV_ERR_CUDA, PIV_ERR_UNSUPPORTED, PIV_ERR_ARGUMENT = 4, 5, 6, 7
PIV_ERR_CANCELLED, PIV_ERR_TIMEOUT = 8, 9
PIV_DTYPE_U8, PIV_DTYPE_U16, PIV_DTYPE_F32 = 0, 1, 2

# Every symbol include/piv_b200.h declares.
EXPORTS = [
    "piv_abi_version", "piv_last_error", "piv_grid", "piv_check_config",
    "piv_analyzer_create", "piv_analyzer_destroy", "piv_num_passes", "piv_output_grid", "piv_pass_grid",
    "piv_analyzer_set_stream", "piv_analyzer_sync", "piv_analyzer_launches", "piv_analyzer_set_profiling",
    "piv_analyzer_profile", "piv_analyzer_autotune", "piv_analyzer_variant", "piv_num_variants",
    "piv_analyzer_set_variant",
    "piv_frame_create", "piv_frame_destroy", "piv_frame_prepare", "piv_frame_prepare_device",
    "piv_frame_set_prepared", "piv_frame_set_prepared_tables", "piv_frame_download", "piv_frame_image_device", "piv_background_device",
    "piv_analyze", "piv_analyze_device", "piv_analyze_traced", "piv_analyze_batch_device",
    "piv_batch_create", "piv_batch_destroy", "piv_batch_input_device", "piv_batch_input_bytes", "piv_batch_run",
    "piv_batch_sync", "piv_batch_outputs_device", "piv_batch_run_host", "piv_batch_kernels", "piv_batch_stream",
    "piv_batch_submit_host", "piv_batch_wait_host", "piv_batch_set_stream", "piv_pipeline_set_background",
    "piv_tc_wait_probe", "piv_batch_set_background",
    "piv_pipeline_create", "piv_pipeline_destroy", "piv_pipeline_submit", "piv_pipeline_wait",
    "piv_place_windows", "piv_correlate_origins", "piv_place_windows_deform", "piv_correlate_deform",
    "piv_validate_field", "piv_flow_stats_device", "piv_temporal_smooth_device", "piv_spatial_smooth_device",
    "piv_tc_selftest", "piv_validate_field_noalloc",
    "piv_server_create", "piv_server_destroy", "piv_server_submit", "piv_server_wait", "piv_server_stats",
    "piv_server_wait_timeout", "piv_server_cancel", "piv_server_fail_next_allocations", "piv_server_set_manual",
    "piv_server_advance", "piv_server_set_fused", "piv_server_reserve",
]


class PivConfigC(ctypes.Structure):
    _fields_ = [
        ("windows", ctypes.POINTER(ctypes.c_int32)),
        ("n_windows", ctypes.c_int32),
        ("overlap", ctypes.c_float),
        ("final_iterations", ctypes.c_int32),
        ("min_mean", ctypes.c_float),
        ("min_std", ctypes.c_float),
        ("ppr_threshold", ctypes.c_float),
        ("median_threshold", ctypes.c_float),
        ("median_eps", ctypes.c_float),
        ("replace", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("deform", ctypes.c_int32),
        ("precision", ctypes.c_int32),
    ]


class PivPreprocessC(ctypes.Structure):
    _fields_ = [
        ("smooth_sigma", ctypes.c_float),
        ("normalize_radius", ctypes.c_int32),
        ("normalize_eps", ctypes.c_float),
        ("clip_percentile", ctypes.c_double),
    ]


class PivGridC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("window", "step", "nx", "ny", "x0", "y0")]


class PivSummaryC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("no_signal", "low_ppr", "median_outliers", "out_of_range", "replaced")]


class PivTraceC(ctypes.Structure):
    _fields_ = [
        ("origins", ctypes.c_void_p), ("raw_dx", ctypes.c_void_p), ("raw_dy", ctypes.c_void_p),
        ("raw_peak_ratio", ctypes.c_void_p), ("raw_flags", ctypes.c_void_p), ("dx", ctypes.c_void_p),
        ("dy", ctypes.c_void_p), ("peak_ratio", ctypes.c_void_p), ("flags", ctypes.c_void_p),
    ]


class PivFlowStatsC(ctypes.Structure):
    _fields_ = [("vorticity_mean", ctypes.c_float), ("vorticity_abs_mean", ctypes.c_float), ("ke_mean", ctypes.c_float),
                ("ke_sum", ctypes.c_float), ("coverage", ctypes.c_float), ("n_usable", ctypes.c_int64),
                ("n_vorticity", ctypes.c_int64)]


class PivServerConfigC(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("memory_budget_bytes", ctypes.c_int64), ("max_in_flight", ctypes.c_int32)]


class PivRequestC(ctypes.Structure):
    _fields_ = [
        ("config", PivConfigC), ("preprocess", PivPreprocessC), ("dtype", ctypes.c_int32),
        ("height", ctypes.c_int64), ("width", ctypes.c_int64), ("frame_a", ctypes.c_void_p),
        ("frame_b", ctypes.c_void_p), ("dx", ctypes.c_void_p), ("dy", ctypes.c_void_p),
        ("peak_ratio", ctypes.c_void_p), ("flags", ctypes.c_void_p),
    ]


class PivServerStatsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("submitted", "admitted", "completed", "failed", "queued", "in_flight",
                                                "memory_in_use_bytes", "steps", "kernel_launches", "cancelled",
                                                "deferred", "last_step_requests", "max_step_requests")]


_lib = None


def load():
    """Loads libpivb200.so (no rebuild, no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libpivb200.so is not built ({LIB_PATH}); run `python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    P = ctypes.POINTER
    sig = {
        "piv_abi_version": ([], i32),
        "piv_last_error": ([], ctypes.c_char_p),
        "piv_grid": ([i64, i64, i64, f32, P(PivGridC)], i32),
        "piv_check_config": ([P(PivConfigC)], i32),
        "piv_analyzer_create": ([P(PivConfigC), P(vp)], i32),
        "piv_analyzer_destroy": ([vp], None),
        "piv_num_passes": ([vp], i32),
        "piv_output_grid": ([vp, i64, i64, P(PivGridC)], i32),
        "piv_pass_grid": ([vp, i64, i64, i32, P(PivGridC)], i32),
        "piv_analyzer_set_stream": ([vp, vp], i32),
        "piv_analyzer_sync": ([vp], i32),
        "piv_analyzer_launches": ([vp], i64),
        "piv_analyzer_set_profiling": ([vp, i32], i32),
        "piv_analyzer_profile": ([vp, i32, P(ctypes.c_double), P(i64)], i32),
        "piv_analyzer_autotune": ([vp, vp, vp], i32),
        "piv_analyzer_variant": ([vp, i32, ctypes.c_char_p, i32], i32),
        "piv_num_variants": ([i32], i32),
        "piv_analyzer_set_variant": ([vp, i32, i32], i32),
        "piv_frame_create": ([vp, i64, i64, P(vp)], i32),
        "piv_frame_destroy": ([vp], None),
        "piv_frame_prepare": ([vp, vp, vp, i32, P(PivPreprocessC), vp], i32),
        "piv_frame_prepare_device": ([vp, vp, vp, i32, P(PivPreprocessC), vp], i32),
        "piv_frame_set_prepared": ([vp, vp, vp, vp], i32),
        "piv_frame_set_prepared_tables": ([vp, vp, vp, vp, vp], i32),
        "piv_frame_download": ([vp, vp, vp], i32),
        "piv_frame_image_device": ([vp], vp),
        "piv_background_device": ([vp, vp, i32, i64, i64, i64, i32, vp], i32),
        "piv_analyze": ([vp, vp, vp, vp, vp, vp, vp, P(PivSummaryC)], i32),
        "piv_analyze_device": ([vp, vp, vp, vp, vp, vp, vp, vp], i32),
        "piv_analyze_traced": ([vp, vp, vp, P(PivTraceC), P(PivSummaryC)], i32),
        "piv_analyze_batch_device": ([vp, vp, vp, i32, vp, vp, vp, vp, vp], i32),
        "piv_batch_create": ([vp, i64, i64, i32, i32, i32, P(PivPreprocessC), P(vp)], i32),
        "piv_batch_destroy": ([vp], None),
        "piv_batch_input_device": ([vp], vp),
        "piv_batch_input_bytes": ([vp], i64),
        "piv_batch_run": ([vp], i32),
        "piv_batch_sync": ([vp], i32),
        "piv_batch_outputs_device": ([vp, P(vp), P(vp), P(vp), P(vp), P(vp)], i32),
        "piv_batch_run_host": ([vp, vp, vp, vp, vp, vp, vp], i32),
        "piv_batch_kernels": ([vp], i64),
        "piv_batch_stream": ([vp], vp),
        "piv_batch_set_stream": ([vp, vp], i32),
        "piv_batch_set_background": ([vp, vp], i32),
        "piv_place_windows": ([vp, i64, i64, P(PivGridC), P(PivGridC), vp, vp, vp], i32),
        "piv_correlate_origins": ([vp, vp, vp, i64, vp, i64, vp, vp, vp, vp], i32),
        "piv_place_windows_deform": ([vp, i64, i64, P(PivGridC), P(PivGridC), vp, vp, vp, vp], i32),
        "piv_correlate_deform": ([vp, vp, vp, P(PivGridC), vp, vp, vp, vp, vp, vp], i32),
        "piv_tc_selftest": ([i32, i32, i32, i32, vp, vp, vp], i32),
        "piv_tc_wait_probe": ([i32, i32, P(i32), P(ctypes.c_float)], i32),
        "piv_batch_submit_host": ([vp, vp, vp, vp, vp, vp], i32),
        "piv_batch_wait_host": ([vp, vp], i32),
        "piv_pipeline_create": ([vp, i64, i64, i32, P(PivPreprocessC), i32, P(vp)], i32),
        "piv_pipeline_destroy": ([vp], None),
        "piv_pipeline_submit": ([vp, vp, vp, vp, vp, vp, vp, P(ctypes.c_uint64)], i32),
        "piv_pipeline_wait": ([vp, ctypes.c_uint64, P(PivSummaryC)], i32),
        "piv_pipeline_set_background": ([vp, vp], i32),
        "piv_flow_stats_device": ([i64, i64, i64, ctypes.c_double, vp, vp, vp, vp, P(PivFlowStatsC), vp], i32),
        "piv_temporal_smooth_device": ([i64, i64, i64, vp, vp, vp, vp, i32, i32, i32, vp, i32, vp, vp, vp, vp], i32),
        "piv_spatial_smooth_device": ([i64, i64, i64, vp, vp, vp, ctypes.c_float, ctypes.c_float, i32, vp, vp, vp, vp],
                                      i32),
        "piv_validate_field": ([vp, i64, i64, vp, vp, vp, vp, vp, vp, vp, P(PivSummaryC)], i32),
        "piv_validate_field_noalloc": ([i64, i64, vp, vp, vp, vp, f32, f32, f32, f32, i32, vp, vp, vp, vp], i32),
        "piv_server_create": ([P(PivServerConfigC), P(vp)], i32),
        "piv_server_destroy": ([vp], None),
        "piv_server_submit": ([vp, P(PivRequestC), P(ctypes.c_uint64)], i32),
        "piv_server_wait": ([vp, ctypes.c_uint64, P(PivSummaryC), P(ctypes.c_double)], i32),
        "piv_server_stats": ([vp, P(PivServerStatsC)], i32),
        "piv_server_wait_timeout": ([vp, ctypes.c_uint64, ctypes.c_double, P(PivSummaryC), P(ctypes.c_double)], i32),
        "piv_server_cancel": ([vp, ctypes.c_uint64], i32),
        "piv_server_fail_next_allocations": ([vp, i32], i32),
        "piv_server_set_manual": ([vp, i32], i32),
        "piv_server_advance": ([vp, i32, ctypes.c_double], i32),
        "piv_server_set_fused": ([vp, i32], i32),
        "piv_server_reserve": ([vp, i64, P(i64)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def last_error():
    return load().piv_last_error().decode(errors="replace")
