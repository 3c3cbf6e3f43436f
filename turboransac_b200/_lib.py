"""ctypes binding of libtbr.so (the C ABI declared in include/tbr.h).

The shared library is built in-tree (turboransac_b200/libtbr.so) by
turboransac_b200.build. There is no fallback: if the library is missing or no
CUDA device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtbr.so")

TBR_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "CANCELLED",
                6: "NOT_READY", 7: "CAPACITY", 8: "INTERNAL"}


class TbrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"tbr error {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class RansacOptionsC(C.Structure):
    _fields_ = [("max_iterations", C.c_uint64), ("min_iterations", C.c_uint64),
                ("dyn_num_trials_mult", C.c_double), ("success_prob", C.c_double),
                ("max_reproj_error", C.c_double), ("max_epipolar_error", C.c_double),
                ("seed", C.c_uint64), ("progressive_sampling", C.c_int32),
                ("max_prosac_iterations", C.c_uint64), ("real_focal_check", C.c_int32),
                ("score_initial_model", C.c_int32)]


class BundleOptionsC(C.Structure):
    _fields_ = [("max_iterations", C.c_uint64), ("loss_type", C.c_int32), ("loss_scale", C.c_double),
                ("gradient_tol", C.c_double), ("step_tol", C.c_double),
                ("initial_lambda", C.c_double), ("min_lambda", C.c_double),
                ("max_lambda", C.c_double), ("verbose", C.c_int32)]


class ExtOptionsC(C.Structure):
    _fields_ = [("honor_options", C.c_int32), ("skip_refine", C.c_int32),
                ("force_samples", C.c_int64), ("max_total_samples", C.c_int64),
                ("seed", C.c_uint64), ("replay_idx", C.c_void_p), ("replay_count", C.c_int64),
                ("hyp_per_thread", C.c_int32), ("chunk_points", C.c_int32),
                ("stop_rule_x86_quirk", C.c_int32), ("points_per_iter", C.c_int32)]


class StatsC(C.Structure):
    _fields_ = [("samples", C.c_int64), ("rounds", C.c_int64), ("hypotheses", C.c_int64),
                ("ransac_inliers", C.c_int64), ("num_inliers", C.c_int64),
                ("inlier_ratio", C.c_double), ("model_score", C.c_double),
                ("best_sample", C.c_int64), ("best_solution", C.c_int32), ("steps", C.c_int32),
                ("candidates_rescored", C.c_int64), ("candidate_overflow", C.c_int32),
                ("lm_iterations", C.c_int32), ("lm_invalid_steps", C.c_int32),
                ("lm_initial_cost", C.c_double), ("lm_cost", C.c_double), ("gpu_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class FrameDescC(C.Structure):
    _fields_ = [("points2D", C.c_void_p), ("points3D", C.c_void_p), ("n", C.c_int64),
                ("K", C.c_double * 4), ("seed", C.c_uint64), ("max_reproj_error", C.c_double)]


class FrameResultC(C.Structure):
    _fields_ = [("q", C.c_double * 4), ("t", C.c_double * 3), ("status", C.c_int32),
                ("pad", C.c_int32), ("stats", StatsC)]


class KernelProfileC(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("total_ms", C.c_double), ("launches", C.c_int64)]


class ServerConfigC(C.Structure):
    _fields_ = [("workspace_budget_bytes", C.c_uint64), ("max_slots", C.c_int32),
                ("max_queue", C.c_int32), ("ransac", RansacOptionsC), ("ext", ExtOptionsC)]


class ServerResultC(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("status", C.c_int32), ("pad", C.c_int32),
                ("q", C.c_double * 4), ("t", C.c_double * 3), ("stats", StatsC),
                ("submit_to_done_ms", C.c_double)]


class TuneEntryC(C.Structure):
    _fields_ = [("hyp_per_thread", C.c_int32), ("points_per_iter", C.c_int32), ("chunk_points", C.c_int32),
                ("pad", C.c_int32), ("ms", C.c_double)]

    def as_dict(self):
        return {"hyp_per_thread": self.hyp_per_thread, "hyp_per_block": 32 * self.hyp_per_thread,
                "points_per_iter": self.points_per_iter, "chunk_points": self.chunk_points, "ms": self.ms}


class ServerStatsC(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("steps", C.c_int64), ("resident_sum", C.c_int64), ("host_stage_ms", C.c_double),
                ("device_wait_ms", C.c_double), ("host_retire_ms", C.c_double), ("host_launch_ms", C.c_double),
                ("pairs_scored", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# Every entry point declared in include/tbr.h.
EXPORTS = [
    "tbr_abi_version", "tbr_last_error", "tbr_default_ransac_options", "tbr_default_bundle_options",
    "tbr_context_create", "tbr_context_destroy", "tbr_estimate_absolute_pose", "tbr_get_inliers", "tbr_estimate_batch_device",
    "tbr_bundle_adjust", "tbr_estimate_batch", "tbr_batch_create", "tbr_batch_run", "tbr_batch_sync",
    "tbr_batch_results", "tbr_batch_destroy", "tbr_batch_profile", "tbr_batch_autotune", "tbr_measure_fp32_peak", "tbr_server_create", "tbr_server_submit",
    "tbr_server_submit_nocopy", "tbr_server_get_stats", "tbr_server_poll", "tbr_server_cancel", "tbr_server_drain", "tbr_server_destroy",
    "tbr_debug_score_samples", "tbr_debug_bounded_wait", "tbr_msac_score_noalloc",
    "tbr_estimate_batch_submit", "tbr_estimate_batch_collect", "tbr_estimate_batch_device_submit",
]


def lib() -> C.CDLL:
    """Load libtbr.so once (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run turboransac_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.tbr_abi_version.restype = C.c_int
    L.tbr_last_error.restype = C.c_char_p
    L.tbr_default_ransac_options.argtypes = [C.POINTER(RansacOptionsC)]
    L.tbr_default_bundle_options.argtypes = [C.POINTER(BundleOptionsC)]
    L.tbr_context_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(vp)]
    L.tbr_context_destroy.argtypes = [vp]
    L.tbr_estimate_absolute_pose.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, C.c_int32,
                                             C.POINTER(RansacOptionsC), C.POINTER(BundleOptionsC),
                                             C.POINTER(ExtOptionsC), vp, vp, vp, C.POINTER(StatsC)]
    L.tbr_get_inliers.argtypes = [vp, vp, vp, vp, vp, C.c_int64, C.c_double, vp, C.POINTER(C.c_int64)]
    L.tbr_bundle_adjust.argtypes = [vp, vp, vp, C.c_int64, vp, vp, vp, C.POINTER(BundleOptionsC), vp,
                                    C.POINTER(ExtOptionsC), C.POINTER(StatsC)]
    L.tbr_estimate_batch.argtypes = [vp, C.POINTER(FrameDescC), C.c_int32, C.POINTER(RansacOptionsC),
                                     C.POINTER(ExtOptionsC), C.POINTER(FrameResultC), vp]
    L.tbr_estimate_batch_device.argtypes = [vp, C.POINTER(FrameDescC), C.c_int32, C.POINTER(RansacOptionsC),
                                            C.POINTER(ExtOptionsC), vp, C.POINTER(FrameResultC), vp]
    L.tbr_estimate_batch_submit.argtypes = [vp, C.POINTER(FrameDescC), C.c_int32, C.POINTER(RansacOptionsC),
                                            C.POINTER(ExtOptionsC), C.POINTER(vp)]
    L.tbr_estimate_batch_collect.argtypes = [vp, C.POINTER(FrameResultC), vp]
    L.tbr_estimate_batch_device_submit.argtypes = [vp, C.POINTER(FrameDescC), C.c_int32,
                                                   C.POINTER(RansacOptionsC), C.POINTER(ExtOptionsC), vp,
                                                   C.POINTER(vp)]
    L.tbr_batch_create.argtypes = [vp, C.POINTER(FrameDescC), C.c_int32, C.POINTER(RansacOptionsC),
                                   C.POINTER(ExtOptionsC), C.POINTER(vp)]
    L.tbr_batch_run.argtypes = [vp]
    L.tbr_batch_sync.argtypes = [vp]
    L.tbr_batch_results.argtypes = [vp, C.POINTER(FrameResultC)]
    L.tbr_batch_destroy.argtypes = [vp]
    L.tbr_batch_profile.argtypes = [vp, C.POINTER(KernelProfileC), C.c_int32, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_uint64)]
    L.tbr_batch_autotune.argtypes = [vp, C.c_int32, C.POINTER(TuneEntryC), C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(TuneEntryC)]
    L.tbr_measure_fp32_peak.argtypes = [vp, C.POINTER(C.c_double)]
    L.tbr_server_create.argtypes = [vp, C.POINTER(ServerConfigC), C.POINTER(vp)]
    L.tbr_server_submit.argtypes = [vp, C.POINTER(FrameDescC), C.POINTER(C.c_uint64)]
    L.tbr_server_submit_nocopy.argtypes = [vp, C.POINTER(FrameDescC), C.POINTER(C.c_uint64)]
    L.tbr_server_get_stats.argtypes = [vp, C.POINTER(ServerStatsC)]
    L.tbr_server_poll.argtypes = [vp, C.POINTER(ServerResultC), C.c_int32, C.POINTER(C.c_int32)]
    L.tbr_server_cancel.argtypes = [vp, C.c_uint64]
    L.tbr_server_drain.argtypes = [vp]
    L.tbr_server_destroy.argtypes = [vp]
    L.tbr_debug_score_samples.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_double, vp, C.c_int64, vp,
                                          vp, vp, vp, C.c_int64, C.POINTER(C.c_int64), vp]
    L.tbr_debug_bounded_wait.argtypes = [vp, C.c_uint32]
    L.tbr_msac_score_noalloc.argtypes = [vp, vp, C.c_int64, vp, C.c_int32, C.c_double, vp, vp, vp]
    for name in EXPORTS:
        fn = getattr(L, name)
        if fn.restype is C.c_int and name not in ("tbr_abi_version",):
            fn.restype = C.c_int
    _lib = L
    return L


def check(status: int) -> None:
    if status != TBR_OK:
        msg = lib().tbr_last_error()
        raise TbrError(status, msg.decode() if msg else "")
