"""ctypes wrapper of the CPU oracle (oracle/libnicp_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product.  The oracle restates the
yorsh87/nicp path in C++ (see nicp_oracle.cpp for the file:line map); its
parity is unpinned because the reference ships no golden vectors.

    REF32 (mode 0)  float, reference operation order, OpenMP partition drops
    F64   (mode 1)  the same algorithm in double, no drops
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnicp_oracle.so")
REF32, F64 = 0, 1


class Camera(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("scaling", C.c_float), ("rows", C.c_int), ("cols", C.c_int),
                ("min_distance", C.c_float), ("max_distance", C.c_float),
                ("baseline", C.c_float), ("alpha", C.c_float)]


class CloudParams(C.Structure):
    _fields_ = [("depth_scale", C.c_float), ("world_radius", C.c_float),
                ("min_image_radius", C.c_int), ("max_image_radius", C.c_int), ("min_points", C.c_int),
                ("curvature_threshold", C.c_float),
                ("pim_flat", C.c_float * 3), ("pim_nonflat", C.c_float * 3), ("pim_curvature_threshold", C.c_float),
                ("nim_flat", C.c_float * 3), ("nim_nonflat", C.c_float * 3), ("nim_curvature_threshold", C.c_float)]


class AlignParams(C.Structure):
    _fields_ = [("inlier_distance_threshold", C.c_float), ("inlier_normal_angular_threshold", C.c_float),
                ("flat_curvature_threshold", C.c_float), ("inlier_curvature_ratio_threshold", C.c_float),
                ("corr_demoted_to_gicp", C.c_int), ("inlier_max_chi2", C.c_float), ("robust_kernel", C.c_int),
                ("z_scaling", C.c_int), ("lin_scale", C.c_float), ("lin_demoted_to_gicp", C.c_int),
                ("outer_iterations", C.c_int), ("inner_iterations", C.c_int), ("lambda_", C.c_float),
                ("translational_min_eigen_ratio", C.c_float), ("rotational_min_eigen_ratio", C.c_float),
                ("threads", C.c_int), ("early_exit_eps", C.c_double), ("row_search_region", C.c_int),
                ("col_search_region", C.c_int)]


class AlignResult(C.Structure):
    _fields_ = [("T", C.c_double * 16), ("error", C.c_double), ("inliers", C.c_int),
                ("num_correspondences", C.c_int), ("translational_ratio", C.c_double),
                ("rotational_ratio", C.c_double), ("solution_valid", C.c_int), ("outer_iterations_run", C.c_int),
                ("omega", C.c_double * 36), ("mean", C.c_double * 6)]


_lib = None
P = C.c_void_p
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


def build():
    """Compiles the oracle with its Makefile (g++ -ffp-contract=off -fopenmp)."""
    r = subprocess.run(["make", "-C", HERE, "-s"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    sig = {
        "orc_convert_u16": (None, [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_float, C.POINTER(C.c_float)]),
        "orc_cloud_build_u16": (P, [C.c_int, C.POINTER(C.c_uint16), C.c_int, C.c_int, C.POINTER(Camera),
                                    C.POINTER(CloudParams), dp, ip]),
        "orc_cloud_build_f32": (P, [C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(Camera),
                                    C.POINTER(CloudParams), dp, ip]),
        "orc_cloud_from_arrays": (P, [C.c_int, C.c_int, dp, dp, dp, dp, dp]),
        "orc_cloud_free": (None, [P]),
        "orc_cloud_size": (C.c_int, [P]),
        "orc_cloud_transform": (None, [P, dp]),
        "orc_depth_scale": (None, [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_float)]),
        "orc_cloud_add": (None, [P, P, dp]),
        "orc_merge": (C.c_int, [C.c_int, P, C.POINTER(Camera), dp, C.c_double, C.c_double]),
        "orc_correspond_nn": (C.c_int, [C.c_int, P, P, dp, C.c_double, C.POINTER(AlignParams), ip]),
        "orc_align_nn": (None, [C.c_int, P, P, dp, C.c_double, C.POINTER(AlignParams), C.c_int,
                                C.POINTER(AlignResult)]),
        "orc_cloud_get": (C.c_int, [P, C.c_int, dp]),
        "orc_projector_matrices": (None, [C.c_int, C.POINTER(Camera), dp, dp, dp]),
        "orc_project": (None, [C.c_int, P, C.POINTER(Camera), dp, ip, dp]),
        "orc_correspond": (C.c_int, [C.c_int, P, P, ip, ip, C.c_int, C.c_int, dp, C.POINTER(AlignParams), ip]),
        "orc_linearize": (None, [C.c_int, P, P, ip, C.c_int, dp, C.POINTER(AlignParams), dp, dp, dp,
                                 C.POINTER(C.c_int)]),
        "orc_align": (None, [C.c_int, P, P, C.POINTER(Camera), dp, dp, dp, C.POINTER(AlignParams), C.c_int,
                             C.POINTER(AlignResult)]),
        "orc_eig3": (None, [C.c_int, dp, dp, dp]),
        "orc_ldlt_solve": (None, [C.c_int, dp, dp, dp]),
        "orc_v2t": (None, [C.c_int, dp, dp]),
        "orc_t2v": (None, [C.c_int, dp, dp]),
        "orc_iso_inverse": (None, [C.c_int, dp, dp]),
        "orc_integral_region": (None, [C.c_int, P, ip, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)


def camera(rows, cols, fx=1.0, fy=1.0, cx=0.5, cy=0.5, scaling=1.0, min_distance=0.01, max_distance=6.0,
           baseline=0.075, alpha=0.1):
    return Camera(fx, fy, cx, cy, scaling, rows, cols, min_distance, max_distance, baseline, alpha)


def cloud_params(**kw):
    p = CloudParams()
    p.depth_scale = 0.001
    p.world_radius = 0.1
    p.min_image_radius, p.max_image_radius, p.min_points = 10, 30, 50
    p.curvature_threshold = 0.02
    p.pim_flat[:] = [1000.0, 0.001, 0.001]
    p.pim_nonflat[:] = [1.0, 0.1, 0.1]
    p.pim_curvature_threshold = 0.02
    p.nim_flat[:] = [1000.0, 0.001, 0.001]
    p.nim_nonflat[:] = [0.1, 1.0, 1.0]
    p.nim_curvature_threshold = 0.02
    for k, v in kw.items():
        if isinstance(getattr(p, k), C.Array):
            getattr(p, k)[:] = v
        else:
            setattr(p, k, v)
    return p


def align_params(**kw):
    p = AlignParams()
    p.inlier_distance_threshold = 1.0
    p.inlier_normal_angular_threshold = float(np.float32(math.cos(np.float32(math.pi / 6))))
    p.flat_curvature_threshold = 0.2
    p.inlier_curvature_ratio_threshold = 1.3
    p.corr_demoted_to_gicp = 0
    p.inlier_max_chi2 = 9e3
    p.robust_kernel = 1
    p.z_scaling = 0
    p.lin_scale = 1.0
    p.lin_demoted_to_gicp = 0
    p.outer_iterations, p.inner_iterations = 10, 1
    p.lambda_ = 1e3
    p.translational_min_eigen_ratio = p.rotational_min_eigen_ratio = 50.0
    p.threads = 1
    p.early_exit_eps = 0.0
    p.row_search_region = p.col_search_region = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Cloud:
    FIELDS = {"points": (0, 4), "normals": (1, 4), "curvature": (2, 1), "omega_p": (3, 9), "omega_n": (4, 9),
              "eigenvalues": (5, 3), "eigenvectors": (6, 9), "stats_n": (7, 1), "gaussian_cov": (8, 9),
              "gaussian_mean": (9, 3)}

    def __init__(self, handle, mode):
        self.h = handle
        self.mode = mode

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_cloud_free(self.h)
            self.h = None

    def __len__(self):
        return load().orc_cloud_size(self.h)

    def get(self, name):
        f, w = self.FIELDS[name]
        n = len(self)
        out = np.zeros(n * w, dtype=np.float64)
        load().orc_cloud_get(self.h, f, out.ctypes.data_as(dp))
        return out.reshape(n, w) if w > 1 else out

    @staticmethod
    def from_arrays(mode, points, normals, curvature, omega_p=None, omega_n=None):
        n = len(points)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(n, 4)
        nrm = np.ascontiguousarray(normals, dtype=np.float64).reshape(n, 4)
        k = np.ascontiguousarray(curvature, dtype=np.float64).reshape(n)
        op = None if omega_p is None else np.ascontiguousarray(omega_p, dtype=np.float64).reshape(n, 9)
        on = None if omega_n is None else np.ascontiguousarray(omega_n, dtype=np.float64).reshape(n, 9)
        h = load().orc_cloud_from_arrays(mode, n, _d(pts), _d(nrm), _d(k), _d(op), _d(on))
        return Cloud(h, mode)


def build_cloud(mode, depth_u16, cam, prm=None, sensor_offset=None):
    """DepthImageConverterIntegralImage::compute; returns (Cloud, index image)."""
    depth = np.ascontiguousarray(depth_u16, dtype=np.uint16)
    rows, cols = depth.shape
    prm = prm or cloud_params()
    index = np.zeros((rows, cols), dtype=np.int32)
    h = load().orc_cloud_build_u16(mode, depth.ctypes.data_as(C.POINTER(C.c_uint16)), rows, cols, C.byref(cam),
                                   C.byref(prm), _d(sensor_offset), index.ctypes.data_as(ip))
    return Cloud(h, mode), index


def build_cloud_f32(mode, depth_f32, cam, prm=None, sensor_offset=None):
    """DepthImageConverterIntegralImage::compute on a float depth image (metres)."""
    depth = np.ascontiguousarray(depth_f32, dtype=np.float32)
    rows, cols = depth.shape
    prm = prm or cloud_params()
    index = np.zeros((rows, cols), dtype=np.int32)
    h = load().orc_cloud_build_f32(mode, depth.ctypes.data_as(C.POINTER(C.c_float)), rows, cols, C.byref(cam),
                                   C.byref(prm), _d(sensor_offset), index.ctypes.data_as(ip))
    return Cloud(h, mode), index


def projector_matrices(mode, cam, T=None):
    K, iK = np.zeros(16), np.zeros(16)
    load().orc_projector_matrices(mode, C.byref(cam), _d(T), K.ctypes.data_as(dp), iK.ctypes.data_as(dp))
    return K.reshape(4, 4), iK.reshape(4, 4)


def _same_mode(mode, *clouds):
    for c in clouds:
        if c.mode != mode:
            raise ValueError("oracle cloud built in mode %d used in mode %d" % (c.mode, mode))


def project(mode, cloud, cam, T=None):
    _same_mode(mode, cloud)
    rows, cols = int(cam.rows * cam.scaling), int(cam.cols * cam.scaling)
    index = np.zeros((rows, cols), dtype=np.int32)
    depth = np.zeros((rows, cols), dtype=np.float64)
    load().orc_project(mode, cloud.h, C.byref(cam), _d(T), index.ctypes.data_as(ip), depth.ctypes.data_as(dp))
    return index, depth


def correspond(mode, ref, cur, ref_index, cur_index, T, prm=None):
    prm = prm or align_params()
    _same_mode(mode, ref, cur)
    rows, cols = ref_index.shape
    pairs = np.zeros(2 * rows * cols, dtype=np.int32)
    ri = np.ascontiguousarray(ref_index, dtype=np.int32)
    ci = np.ascontiguousarray(cur_index, dtype=np.int32)
    k = load().orc_correspond(mode, ref.h, cur.h, ri.ctypes.data_as(ip), ci.ctypes.data_as(ip), rows, cols, _d(T),
                              C.byref(prm), pairs.ctypes.data_as(ip))
    return pairs[:2 * k].reshape(k, 2)


def linearize(mode, ref, cur, pairs, T, prm=None):
    prm = prm or align_params()
    _same_mode(mode, ref, cur)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    H, b, err = np.zeros(36), np.zeros(6), np.zeros(1)
    inl = C.c_int(0)
    load().orc_linearize(mode, ref.h, cur.h, pairs.ctypes.data_as(ip), len(pairs), _d(T), C.byref(prm),
                         H.ctypes.data_as(dp), b.ctypes.data_as(dp), err.ctypes.data_as(dp), C.byref(inl))
    return H.reshape(6, 6), b, float(err[0]), inl.value


def depth_scale(depth_f32, step, max_depth_cov=0.01):
    """DepthImage_scale (imageutils.cpp:6-37) of a float depth image."""
    d = np.ascontiguousarray(depth_f32, dtype=np.float32)
    rows, cols = d.shape
    out = np.zeros((rows // step, cols // step), np.float32)
    load().orc_depth_scale(d.ctypes.data_as(C.POINTER(C.c_float)), rows, cols, step, max_depth_cov,
                           out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def convert_u16(depth_u16, scale=0.001):
    """DepthImage_convert_16UC1_to_32FC1 (imageutils.cpp:85-99)."""
    d = np.ascontiguousarray(depth_u16, dtype=np.uint16)
    out = np.zeros(d.shape, np.float32)
    load().orc_convert_u16(d.ctypes.data_as(C.POINTER(C.c_uint16)), d.shape[0], d.shape[1], np.float32(scale),
                           out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def correspond_nn(mode, ref, cur, T, normal_scaling=1.0, prm=None):
    """CorrespondenceFinderNN::compute with an exact nearest neighbour."""
    prm = prm or align_params()
    _same_mode(mode, ref, cur)
    pairs = np.zeros(2 * max(len(ref), 1), dtype=np.int32)
    k = load().orc_correspond_nn(mode, ref.h, cur.h, _d(T), normal_scaling, C.byref(prm), pairs.ctypes.data_as(ip))
    return pairs[:2 * k].reshape(k, 2)


def align_nn(mode, ref, cur, guess=None, normal_scaling=1.0, prm=None, statistics=False):
    """AlignerNN::align (alignernn.cpp:21-118)."""
    prm = prm or align_params()
    _same_mode(mode, ref, cur)
    r = AlignResult()
    load().orc_align_nn(mode, ref.h, cur.h, _d(guess), normal_scaling, C.byref(prm), 1 if statistics else 0,
                        C.byref(r))
    return dict(T=np.array(r.T).reshape(4, 4), error=r.error, inliers=r.inliers,
                num_correspondences=r.num_correspondences, translational_ratio=r.translational_ratio,
                rotational_ratio=r.rotational_ratio, solution_valid=r.solution_valid)


def cloud_transform(cloud, T):
    """Cloud::transformInPlace (cloud.cpp:191-204)."""
    load().orc_cloud_transform(cloud.h, _d(T))


def cloud_add(dst, src, T):
    """Cloud::add (cloud.cpp:163-189): src is transformed in place by T and
    appended to dst."""
    _same_mode(dst.mode, src)
    load().orc_cloud_add(dst.h, src.h, _d(T))


def merge(mode, cloud, cam, T, distance_threshold=0.1, max_point_depth=10.0):
    """Merger::merge (merger.cpp:15-109); returns the number of removed points."""
    _same_mode(mode, cloud)
    return load().orc_merge(mode, cloud.h, C.byref(cam), _d(T), distance_threshold, max_point_depth)


def align(mode, ref, cur, cam, guess=None, ref_offset=None, cur_offset=None, prm=None, statistics=False):
    prm = prm or align_params()
    _same_mode(mode, ref, cur)
    r = AlignResult()
    load().orc_align(mode, ref.h, cur.h, C.byref(cam), _d(guess), _d(ref_offset), _d(cur_offset), C.byref(prm),
                     1 if statistics else 0, C.byref(r))
    return dict(T=np.array(r.T).reshape(4, 4), error=r.error, inliers=r.inliers,
                num_correspondences=r.num_correspondences, translational_ratio=r.translational_ratio,
                rotational_ratio=r.rotational_ratio, solution_valid=r.solution_valid,
                outer_iterations_run=r.outer_iterations_run, omega=np.array(r.omega).reshape(6, 6),
                mean=np.array(r.mean))


def eig3(mode, A6):
    lam, U = np.zeros(3), np.zeros(9)
    load().orc_eig3(mode, _d(np.asarray(A6, float)), lam.ctypes.data_as(dp), U.ctypes.data_as(dp))
    return lam, U.reshape(3, 3)


def ldlt_solve(mode, A, b):
    x = np.zeros(6)
    load().orc_ldlt_solve(mode, _d(np.asarray(A, float).reshape(36)), _d(np.asarray(b, float)), x.ctypes.data_as(dp))
    return x


def v2t(mode, x):
    T = np.zeros(16)
    load().orc_v2t(mode, _d(np.asarray(x, float)), T.ctypes.data_as(dp))
    return T.reshape(4, 4)


def t2v(mode, T):
    x = np.zeros(6)
    load().orc_t2v(mode, _d(np.asarray(T, float).reshape(16)), x.ctypes.data_as(dp))
    return x


def iso_inverse(mode, T):
    o = np.zeros(16)
    load().orc_iso_inverse(mode, _d(np.asarray(T, float).reshape(16)), o.ctypes.data_as(dp))
    return o.reshape(4, 4)


def integral_region(mode, cloud, index, xmin, xmax, ymin, ymax):
    _same_mode(mode, cloud)
    index = np.ascontiguousarray(index, dtype=np.int32)
    rows, cols = index.shape
    out = np.zeros(10)
    load().orc_integral_region(mode, cloud.h, index.ctypes.data_as(ip), rows, cols, xmin, xmax, ymin, ymax,
                               out.ctypes.data_as(dp))
    return out
