"""ctypes binding of libaw_b200.so (the C ABI declared in include/anchorwave_b200.h).

There is no fallback: if the shared library is missing or cannot be loaded, importing
this module raises, so no caller can silently run a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaw_b200.so")


class KswExtz(C.Structure):
    """ksw_extz_t (minimap2/ksw2.h:40-50); identical layout in include/anchorwave_b200.h."""
    _fields_ = [("max", C.c_uint32, 31), ("zdropped", C.c_uint32, 1),
                ("max_q", C.c_int), ("max_t", C.c_int), ("mqe", C.c_int), ("mqe_t", C.c_int),
                ("mte", C.c_int), ("mte_q", C.c_int), ("score", C.c_int),
                ("m_cigar", C.c_int), ("n_cigar", C.c_int), ("reach_end", C.c_int),
                ("stopped", C.c_int), ("cigar", C.POINTER(C.c_uint32))]


# Every symbol the header declares; tests check that the library exports each one.
EXPORTS = [
    "ksw_extd2_gpu", "ksw_extd2_singletrack_gpu", "ksw_extd2_singletrack_sse_gpu", "aw_ksw_extd2_batch",
    "aw_ksw_plan_new", "aw_ksw_plan_upload", "aw_ksw_plan_execute", "aw_ksw_plan_download",
    "aw_ksw_plan_stats", "aw_ksw_plan_routes", "aw_ksw_plan_timing", "aw_ksw_plan_graph", "aw_ksw_plan_free",
    "aw_set_traceback_budget", "aw_set_tuning", "aw_set_band_columns", "aw_set_full_pair_routing",
    "aw_set_wfa_wide", "aw_set_wfa_long", "wavefront_gpu_last_launches", "aw_release_thread_buffers",
    "aw_ksw_set_deadline", "aw_ksw_set_stop_antidiagonal", "aw_last_error", "aw_device_count",
    "aw_int32_peak_ops", "aw_int16x2_peak_ops", "aw_ksw_extd2_device_noalloc", "aw_cigar_rows_batch",
    "wavefront_aligner_new_gpu", "wavefront_aligner_delete_gpu", "wavefront_align_gpu", "wavefront_gpu_cigar",
    "wavefront_align_batch_gpu", "wavefront_gpu_memory", "aw_sequence_summary_batch",
    "aw_sequence_summary_sketches", "aw_sequence_summary_sketch_view", "aw_serve_open", "aw_serve_submit", "aw_serve_poll", "aw_serve_stats",
    "aw_serve_result_free", "aw_serve_close", "wavefront_aligner_new_wfa2_gpu", "wavefront_align_wfa2_gpu",
    "wavefront_aligner_delete_wfa2_gpu", "wavefront_aligner_attr_default_gpu", "aw_align_score_certified_batch",
    "aw_certified_result_free", "aw_align_sliding_window_batch", "aw_window_result_free", "aw_serve_submit_route",
]


class CertResultC(C.Structure):
    """aw_certified_result_t (include/anchorwave_b200.h)."""
    _fields_ = [("status", C.c_int), ("score", C.c_int64), ("optimal_score", C.c_int64),
                ("final_band_width", C.c_int64), ("traceback_attempts", C.c_int64),
                ("alignment_q", C.c_void_p), ("alignment_d", C.c_void_p), ("alignment_len", C.c_int64),
                ("best_effort_q", C.c_void_p), ("best_effort_d", C.c_void_p), ("best_effort_len", C.c_int64)]


class WindowResultC(C.Structure):
    """aw_window_result_t (include/anchorwave_b200.h)."""
    _fields_ = [("score", C.c_int64), ("alignment_q", C.c_void_p), ("alignment_d", C.c_void_p),
                ("alignment_len", C.c_int64)]


class ServeConfig(C.Structure):
    """aw_serve_config_t (include/anchorwave_b200.h)."""
    _fields_ = [("slots", C.c_int), ("max_batch", C.c_int), ("hbm_budget", C.c_int64), ("m", C.c_int8),
                ("mat", C.c_int8 * 64), ("q", C.c_int8), ("e", C.c_int8), ("q2", C.c_int8), ("e2", C.c_int8),
                ("wfa_x", C.c_int), ("wfa_o1", C.c_int), ("wfa_e1", C.c_int), ("wfa_o2", C.c_int),
                ("wfa_e2", C.c_int)]


class ServeRoute(C.Structure):
    """aw_serve_route_t."""
    _fields_ = [("method", C.c_int), ("band", C.c_int), ("band_max", C.c_int), ("window", C.c_int64),
                ("predicted_bytes", C.c_int64)]


class ServeResult(C.Structure):
    """aw_serve_result_t."""
    _fields_ = [("id", C.c_uint64), ("method", C.c_int), ("status", C.c_int), ("ez", KswExtz),
                ("wfa_score", C.c_int), ("n_ops", C.c_int), ("ops", C.c_void_p), ("latency_s", C.c_double)]


class ServeStats(C.Structure):
    """aw_serve_stats_t."""
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("micro_batches", C.c_uint64),
                ("queued", C.c_uint64), ("inflight_bytes", C.c_int64), ("latency_p50_s", C.c_double),
                ("latency_p99_s", C.c_double), ("elapsed_s", C.c_double)]


class WfaAttr(C.Structure):
    """wavefront_gpu_attr_t (include/anchorwave_b200.h)."""
    _fields_ = [("mismatch", C.c_int), ("gap_opening1", C.c_int), ("gap_extension1", C.c_int),
                ("gap_opening2", C.c_int), ("gap_extension2", C.c_int), ("singletrack", C.c_int),
                ("memory_mode", C.c_int), ("max_memory_abort", C.c_int64)]


def _load(path: str = LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with `python -m anchorwave_b200.build`")
    lib = C.CDLL(path)
    vp, i8, i32, i64 = C.c_void_p, C.c_int8, C.c_int, C.c_int64
    ksw_args = [vp, i32, vp, i32, vp, i8, vp, i8, i8, i8, i8, i32, i32, i32, i32, C.POINTER(KswExtz)]
    lib.ksw_extd2_gpu.argtypes = ksw_args
    lib.ksw_extd2_gpu.restype = None
    lib.ksw_extd2_singletrack_gpu.argtypes = ksw_args
    lib.ksw_extd2_singletrack_gpu.restype = None
    lib.ksw_extd2_singletrack_sse_gpu.argtypes = ksw_args
    lib.ksw_extd2_singletrack_sse_gpu.restype = None
    lib.aw_ksw_extd2_batch.argtypes = [i32, vp, vp, vp, vp, vp, i8, vp, i8, i8, i8, i8, i32, i32, i32, vp]
    lib.aw_ksw_extd2_batch.restype = i32
    lib.aw_ksw_plan_new.argtypes = [i32, vp, vp, vp, i8, vp, i8, i8, i8, i8, i32, i32, i32]
    lib.aw_ksw_plan_new.restype = vp
    lib.aw_ksw_plan_upload.argtypes = [vp, vp, vp]
    lib.aw_ksw_plan_upload.restype = i32
    lib.aw_ksw_plan_execute.argtypes = [vp, C.POINTER(C.c_float)]
    lib.aw_ksw_plan_execute.restype = i32
    lib.aw_ksw_plan_download.argtypes = [vp, vp]
    lib.aw_ksw_plan_download.restype = i32
    lib.aw_ksw_plan_stats.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(i32)]
    lib.aw_ksw_plan_stats.restype = i32
    lib.aw_ksw_plan_routes.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    lib.aw_ksw_plan_routes.restype = i32
    lib.aw_ksw_plan_timing.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.aw_ksw_plan_timing.restype = i32
    lib.aw_ksw_plan_free.argtypes = [vp]
    lib.aw_ksw_plan_free.restype = None
    lib.aw_set_traceback_budget.argtypes = [i64]
    lib.aw_set_traceback_budget.restype = None
    lib.aw_set_tuning.argtypes = [i32, i32]
    lib.aw_set_tuning.restype = None
    lib.aw_set_band_columns.argtypes = [i32]
    lib.aw_set_band_columns.restype = None
    lib.aw_set_wfa_wide.argtypes = [i32, i32, i32]
    lib.aw_set_wfa_wide.restype = None
    lib.aw_set_wfa_long.argtypes = [i32]
    lib.aw_set_wfa_long.restype = None
    lib.wavefront_gpu_last_launches.argtypes = [C.c_void_p, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    lib.wavefront_gpu_last_launches.restype = i32
    lib.aw_set_full_pair_routing.argtypes = [i32]
    lib.aw_set_full_pair_routing.restype = None
    lib.aw_release_thread_buffers.argtypes = []
    lib.aw_release_thread_buffers.restype = None
    lib.aw_ksw_set_deadline.argtypes = [C.c_double]
    lib.aw_ksw_set_deadline.restype = None
    lib.aw_ksw_set_stop_antidiagonal.argtypes = [i32, i32]
    lib.aw_ksw_set_stop_antidiagonal.restype = None
    lib.aw_last_error.argtypes = []
    lib.aw_last_error.restype = C.c_char_p
    lib.aw_device_count.argtypes = []
    lib.aw_device_count.restype = i32
    lib.aw_ksw_plan_graph.argtypes = [vp]
    lib.aw_ksw_plan_graph.restype = i32
    lib.aw_cigar_rows_batch.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64]
    lib.aw_cigar_rows_batch.restype = i32
    lib.aw_align_score_certified_batch.argtypes = [i32, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32,
                                                   C.c_double, vp, C.POINTER(CertResultC)]
    lib.aw_align_score_certified_batch.restype = i32
    lib.aw_certified_result_free.argtypes = [C.POINTER(CertResultC)]
    lib.aw_certified_result_free.restype = None
    lib.aw_align_sliding_window_batch.argtypes = [i32, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, i32,
                                                  C.POINTER(WindowResultC)]
    lib.aw_align_sliding_window_batch.restype = i32
    lib.aw_window_result_free.argtypes = [C.POINTER(WindowResultC)]
    lib.aw_window_result_free.restype = None
    lib.aw_int32_peak_ops.argtypes = []
    lib.aw_int32_peak_ops.restype = C.c_double
    lib.aw_int16x2_peak_ops.argtypes = []
    lib.aw_int16x2_peak_ops.restype = C.c_double
    lib.aw_ksw_extd2_device_noalloc.argtypes = [i32, vp, i32, vp, i8, vp, i8, i8, i8, i8, i32, vp, vp, i32, vp]
    lib.aw_ksw_extd2_device_noalloc.restype = i32
    lib.wavefront_aligner_new_gpu.argtypes = [C.POINTER(WfaAttr)]
    lib.wavefront_aligner_new_gpu.restype = vp
    lib.wavefront_aligner_delete_gpu.argtypes = [vp]
    lib.wavefront_aligner_delete_gpu.restype = None
    lib.wavefront_align_gpu.argtypes = [vp, C.c_char_p, i32, C.c_char_p, i32]
    lib.wavefront_align_gpu.restype = i32
    lib.wavefront_gpu_cigar.argtypes = [vp, C.POINTER(C.c_char_p), C.POINTER(i32), C.POINTER(i32)]
    lib.wavefront_gpu_cigar.restype = i32
    lib.wavefront_align_batch_gpu.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, C.POINTER(C.c_float)]
    lib.wavefront_align_batch_gpu.restype = i32
    lib.wavefront_gpu_memory.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    lib.wavefront_gpu_memory.restype = i32
    lib.aw_sequence_summary_batch.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_float)]
    lib.aw_sequence_summary_batch.restype = i32
    lib.aw_sequence_summary_sketches.argtypes = [vp, vp, i64]
    lib.aw_sequence_summary_sketches.restype = i64
    lib.aw_sequence_summary_sketch_view.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    lib.aw_sequence_summary_sketch_view.restype = i64
    lib.aw_serve_open.argtypes = [C.POINTER(ServeConfig)]
    lib.aw_serve_open.restype = vp
    lib.aw_serve_submit.argtypes = [vp, C.c_uint64, i32, i32, C.c_char_p, i32, C.c_char_p, i32]
    lib.aw_serve_submit.restype = i32
    lib.aw_serve_submit_route.argtypes = [vp, C.c_uint64, C.POINTER(ServeRoute), C.c_char_p, i32, C.c_char_p, i32]
    lib.aw_serve_submit_route.restype = i32
    lib.aw_serve_poll.argtypes = [vp, C.POINTER(ServeResult), i32, i32]
    lib.aw_serve_poll.restype = i32
    lib.aw_serve_stats.argtypes = [vp, C.POINTER(ServeStats)]
    lib.aw_serve_stats.restype = i32
    lib.aw_serve_result_free.argtypes = [C.POINTER(ServeResult)]
    lib.aw_serve_result_free.restype = None
    lib.aw_serve_close.argtypes = [vp]
    lib.aw_serve_close.restype = None
    for name in EXPORTS:
        getattr(lib, name)  # raises AttributeError if a declared symbol is missing
    return lib


lib = _load()
libc = C.CDLL(None)
libc.free.argtypes = [C.c_void_p]
libc.free.restype = None


def last_error() -> str:
    msg = lib.aw_last_error()
    return msg.decode() if msg else ""


class AwError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != 0:
        raise AwError(f"{what} failed ({rc}): {last_error()}")
