"""ctypes binding of include/nicp_gpu.h (libnicp_b200.so).

This is the Python side of the drop-in boundary: every C entry point is
declared here with its exact signature.  Loading fails loudly when the
library has not been built; there is no fallback implementation.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnicp_b200.so")

NICP_OK, NICP_EINVAL, NICP_ENOMEM, NICP_EBUDGET, NICP_ETIMEOUT, NICP_ECUDA, NICP_ESTATE = range(7)
NICP_MOMENTS_F64, NICP_MOMENTS_F32, NICP_MOMENTS_TWOFLOAT = range(3)
KERNELS = ["unproject", "moments_bands", "moments_sweep", "stats_omega", "zbuffer", "resolve", "corr_lin",
           "corr_list", "lin_list", "solve", "transform"]
K = {name: i for i, name in enumerate(KERNELS)}

F3 = C.c_float * 3
F16 = C.c_float * 16
D16 = C.c_double * 16


class Camera(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("scaling", C.c_float), ("rows", C.c_int), ("cols", C.c_int),
                ("min_distance", C.c_float), ("max_distance", C.c_float),
                ("baseline", C.c_float), ("alpha", C.c_float)]


class CloudParams(C.Structure):
    _fields_ = [("depth_scale", C.c_float), ("world_radius", C.c_float),
                ("min_image_radius", C.c_int), ("max_image_radius", C.c_int), ("min_points", C.c_int),
                ("curvature_threshold", C.c_float),
                ("pim_flat", F3), ("pim_nonflat", F3), ("pim_curvature_threshold", C.c_float),
                ("nim_flat", F3), ("nim_nonflat", F3), ("nim_curvature_threshold", C.c_float),
                ("moments_precision", C.c_int), ("keep_stats", C.c_int), ("keep_gaussians", C.c_int)]


class CorrParams(C.Structure):
    _fields_ = [("inlier_distance_threshold", C.c_float), ("inlier_normal_angular_threshold", C.c_float),
                ("flat_curvature_threshold", C.c_float), ("inlier_curvature_ratio_threshold", C.c_float),
                ("demoted_to_gicp", C.c_int), ("parity_threads", C.c_int), ("row_search_region", C.c_int),
                ("col_search_region", C.c_int)]


class LinParams(C.Structure):
    _fields_ = [("inlier_max_chi2", C.c_float), ("robust_kernel", C.c_int), ("z_scaling", C.c_int),
                ("scale", C.c_float), ("demoted_to_gicp", C.c_int), ("cross_block_f32", C.c_int)]


class AlignParams(C.Structure):
    _fields_ = [("outer_iterations", C.c_int), ("inner_iterations", C.c_int), ("lambda_", C.c_float),
                ("min_inliers", C.c_int), ("translational_min_eigen_ratio", C.c_float),
                ("rotational_min_eigen_ratio", C.c_float), ("compute_statistics", C.c_int),
                ("early_exit_eps", C.c_double)]


class AlignResult(C.Structure):
    _fields_ = [("T", D16), ("error", C.c_float), ("inliers", C.c_int), ("num_correspondences", C.c_int),
                ("outer_iterations_run", C.c_int), ("translational_ratio", C.c_double),
                ("rotational_ratio", C.c_double), ("solution_valid", C.c_int), ("status", C.c_int),
                ("omega", C.c_double * 36), ("mean", C.c_double * 6)]


class ServerParams(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_batch", C.c_int), ("workers", C.c_int),
                ("keyframe_min_inlier_ratio", C.c_float), ("cloud", CloudParams), ("corr", CorrParams),
                ("lin", LinParams), ("align", AlignParams)]


class ServerResult(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("stream_id", C.c_int), ("status", C.c_int), ("T", D16),
                ("error", C.c_float), ("inliers", C.c_int), ("keyframe_points", C.c_int),
                ("keyframe_replaced", C.c_int), ("batch_size", C.c_int), ("latency_ms", C.c_double),
                ("queue_ms", C.c_double)]


P = C.c_void_p
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "nicp_default_camera": (None, [C.POINTER(Camera)]),
    "nicp_default_cloud_params": (None, [C.POINTER(CloudParams)]),
    "nicp_default_corr_params": (None, [C.POINTER(CorrParams)]),
    "nicp_default_lin_params": (None, [C.POINTER(LinParams)]),
    "nicp_default_align_params": (None, [C.POINTER(AlignParams)]),
    "nicp_ctx_create": (C.c_int, [C.c_int, P, C.POINTER(P)]),
    "nicp_ctx_destroy": (C.c_int, [P]),
    "nicp_ctx_last_error": (C.c_char_p, [P]),
    "nicp_ctx_synchronize": (C.c_int, [P]),
    "nicp_ctx_stream": (P, [P]),
    "nicp_ctx_device_bytes": (C.c_size_t, [P]),
    "nicp_ctx_set_profiling": (C.c_int, [P, C.c_int]),
    "nicp_ctx_kernel_launches": (C.c_ulonglong, [P]),
    "nicp_ctx_set_autotune": (C.c_int, [P, C.c_int]),
    "nicp_ctx_launch_shape": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nicp_ctx_transfer_bytes": (C.c_int, [P, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    "nicp_ctx_read_profile": (C.c_int, [P, C.c_int, f64p, C.POINTER(C.c_int)]),
    "nicp_kernel_name": (C.c_char_p, [C.c_int]),
    "nicp_cloud_create": (C.c_int, [P, C.POINTER(P)]),
    "nicp_cloud_destroy": (C.c_int, [P]),
    "nicp_cloud_size": (C.c_int, [P, C.POINTER(C.c_int)]),
    "nicp_cloud_normal_count": (C.c_int, [P, C.POINTER(C.c_int)]),
    "nicp_cloud_download": (C.c_int, [P, f32p, f32p, f32p, f32p, f32p, f32p, f32p]),
    "nicp_cloud_download_gaussians": (C.c_int, [P, f32p, f32p]),
    "nicp_cloud_download_stats": (C.c_int, [P, f32p, f32p, f32p, i32p]),
    "nicp_cloud_upload": (C.c_int, [P, C.c_int, f32p, f32p, f32p, f32p, f32p]),
    "nicp_cloud_transform": (C.c_int, [P, f32p]),
    "nicp_cloud_add": (C.c_int, [P, P, f32p]),
    "nicp_correspond_nn": (C.c_int, [P, P, P, f32p, C.c_float, C.POINTER(CorrParams), i32p, C.POINTER(C.c_int)]),
    "nicp_align_nn": (C.c_int, [P, P, P, f32p, C.c_float, C.POINTER(CorrParams), C.POINTER(LinParams),
                                C.POINTER(AlignParams), C.POINTER(AlignResult)]),
    "nicp_cloud_save": (C.c_int, [P, C.c_char_p, f32p, C.c_int, C.c_int]),
    "nicp_cloud_load": (C.c_int, [P, C.c_char_p, C.POINTER(CloudParams), f32p, C.POINTER(C.c_int)]),
    "nicp_trajectory_line": (C.c_int, [C.c_char_p, f32p, C.c_char_p, C.c_size_t]),
    "nicp_depth_scale": (C.c_int, [P, P, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_float, C.c_int, C.c_float,
                                   P, C.c_int]),
    "nicp_merge": (C.c_int, [P, P, C.POINTER(Camera), f32p, C.c_float, C.c_float, C.POINTER(C.c_int)]),
    "nicp_cloud_from_depth_u16": (C.c_int, [P, P, C.c_int, C.c_int, C.c_size_t, C.c_int, C.POINTER(Camera),
                                            C.POINTER(CloudParams), f32p, P, i32p]),
    "nicp_cloud_from_depth_f32": (C.c_int, [P, P, C.c_int, C.c_int, C.c_size_t, C.c_int, C.POINTER(Camera),
                                            C.POINTER(CloudParams), f32p, P, i32p]),
    "nicp_projector_matrices": (C.c_int, [C.POINTER(Camera), f32p, f32p, f32p]),
    "nicp_unproject": (C.c_int, [P, f32p, C.c_int, C.c_int, C.POINTER(Camera), f32p, f32p, i32p,
                                 C.POINTER(C.c_int)]),
    "nicp_project_intervals": (C.c_int, [P, f32p, C.c_int, C.c_int, C.POINTER(Camera), C.c_float, i32p]),
    "nicp_project": (C.c_int, [P, P, C.POINTER(Camera), f32p, i32p, f32p]),
    "nicp_correspond": (C.c_int, [P, P, P, i32p, i32p, C.c_int, C.c_int, f32p, C.POINTER(CorrParams), i32p,
                                  C.POINTER(C.c_int)]),
    "nicp_linearize": (C.c_int, [P, P, P, i32p, C.c_int, f32p, C.POINTER(LinParams), C.c_int, f64p, f64p,
                                 f64p, C.POINTER(C.c_int)]),
    "nicp_linearize_noalloc": (C.c_int, [P, P, P, P, C.c_int, f32p, C.POINTER(LinParams), C.c_int, P]),
    "nicp_align": (C.c_int, [P, P, P, C.POINTER(Camera), f32p, f32p, f32p, C.POINTER(CorrParams),
                             C.POINTER(LinParams), C.POINTER(AlignParams), C.POINTER(AlignResult)]),
    "nicp_build_batch": (C.c_int, [P, C.c_int, C.POINTER(P), i32p, i32p, C.c_int, C.POINTER(Camera),
                                   C.POINTER(CloudParams), C.POINTER(P)]),
    "nicp_align_batch": (C.c_int, [P, C.c_int, C.POINTER(P), C.POINTER(P), C.POINTER(Camera), f32p,
                                   C.POINTER(CorrParams), C.POINTER(LinParams), C.POINTER(AlignParams),
                                   C.POINTER(AlignResult)]),
    "nicp_default_server_params": (None, [C.POINTER(ServerParams)]),
    "nicp_server_create": (C.c_int, [C.c_int, C.POINTER(ServerParams), C.POINTER(P)]),
    "nicp_server_submit": (C.c_int, [P, C.c_int, C.c_uint64, P, C.c_int, C.c_int, C.POINTER(Camera)]),
    "nicp_server_poll": (C.c_int, [P, C.POINTER(ServerResult), C.c_int, C.POINTER(C.c_int), C.c_int]),
    "nicp_server_status": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "nicp_server_destroy": (C.c_int, [P]),
}

_lib = None


def load():
    """Loads libnicp_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libnicp_b200.so is missing: run `python -m nicp_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NicpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("nicp error %d: %s" % (code, msg))
        self.code = code


def check(rc, ctx=None):
    if rc != NICP_OK:
        msg = load().nicp_ctx_last_error(ctx).decode() if ctx else ""
        raise NicpError(rc, msg)


def fptr(a):
    return a.ctypes.data_as(f32p) if a is not None else None


def dptr(a):
    return a.ctypes.data_as(f64p) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(i32p) if a is not None else None


def f16(T):
    """4x4 transform -> contiguous float32 row-major array (or None)."""
    if T is None:
        return None
    return np.ascontiguousarray(np.asarray(T, dtype=np.float32).reshape(4, 4))


NICP_LINEARIZE_NOALLOC_MAX_PAIRS = 1048576  # include/nicp_gpu.h
