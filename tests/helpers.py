"""Shared helpers of the parity tests: the same synthetic inputs fed to the
CUDA path (through the C ABI) and to the CPU oracle."""
import math

import numpy as np

from nicp_b200 import _lib as L
from nicp_b200 import api, synth
from oracle import oracle as O


def cams(cam):
    """(product Camera, oracle Camera) for a synth camera dict."""
    pc = L.Camera()
    pc.fx, pc.fy, pc.cx, pc.cy = cam["fx"], cam["fy"], cam["cx"], cam["cy"]
    pc.scaling = 1.0
    pc.rows, pc.cols = cam["rows"], cam["cols"]
    pc.min_distance, pc.max_distance = cam.get("min_distance", 0.01), cam.get("max_distance", 6.0)
    pc.baseline, pc.alpha = 0.075, 0.1
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"],
                  min_distance=pc.min_distance, max_distance=pc.max_distance)
    return pc, oc


def projector(cam, ctx=None):
    p = api.PinholePointProjector(ctx)
    p.setCameraMatrix([[cam["fx"], 0, cam["cx"]], [0, cam["fy"], cam["cy"]], [0, 0, 1]])
    p.setImageSize(cam["rows"], cam["cols"])
    p.setMinDistance(cam.get("min_distance", 0.01))
    p.setMaxDistance(cam.get("max_distance", 6.0))
    return p


def converter(cam, ctx=None, keep_stats=False, precision=L.NICP_MOMENTS_F64):
    proj = projector(cam, ctx)
    stats = api.StatsCalculatorIntegralImage()
    stats.momentsPrecision = precision
    conv = api.DepthImageConverterIntegralImage(proj, stats, api.PointInformationMatrixCalculator(),
                                                api.NormalInformationMatrixCalculator())
    conv.keepStats = keep_stats
    return proj, conv


def gpu_cloud(ctx, conv, depth, keep_index=True):
    c = api.Cloud(ctx)
    conv.compute(c, depth, keep_index=keep_index)
    return c, conv.indexImage()


def oracle_cloud_from_gpu(mode, gpu_dl):
    """An oracle cloud holding exactly the GPU cloud's float values."""
    n = len(gpu_dl["points"])
    return O.Cloud.from_arrays(mode, gpu_dl["points"].astype(np.float64), gpu_dl["normals"].astype(np.float64),
                               gpu_dl["curvature"].astype(np.float64),
                               gpu_dl["omega_p"].reshape(n, 9).astype(np.float64),
                               gpu_dl["omega_n"].reshape(n, 9).astype(np.float64))


def float_T(T):
    return np.asarray(T, np.float32).astype(np.float64)


def perturb(seed, deg=1.0, m=0.02):
    rng = np.random.default_rng(seed)
    return synth.random_offset(rng, deg, deg, m, m)


def rot_err(Ta, Tb):
    return synth.pose_error(np.asarray(Ta, float), np.asarray(Tb, float))


def angle_between(a, b):
    c = np.clip(np.abs(np.sum(a * b, axis=1)) / (np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1) + 1e-300), 0, 1)
    return np.arccos(c)


def deg(x):
    return math.degrees(x)


def radius_image(depth_u16, cam, dtype, world_radius=0.1, depth_scale=0.001):
    """Interval radius per pixel (pinholepointprojector.h:293-302) evaluated in
    float32 (the reference and the CUDA path) or float64 (the FP64 oracle)."""
    t = np.dtype(dtype).type
    u = depth_u16.astype(np.int64)
    # both start from the float DepthImage (imageutils.cpp:85-99); FP64 promotes it
    d = (np.float32(depth_scale) * u.astype(np.float32)).astype(dtype)
    d = np.where(u == 0, t(0), d)
    R = t(np.float32(world_radius))
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = t(1) / d
        a = (t(np.float32(cam["fx"])) * R) * inv
        b = (t(np.float32(cam["fy"])) * R) * inv
        m = np.where(a < b, b, a)
        lo, hi = t(np.float32(cam.get("min_distance", 0.01))), t(np.float32(cam.get("max_distance", 6.0)))
        r = np.where((d < lo) | (d > hi), -1, np.trunc(np.nan_to_num(m, posinf=0, neginf=0))).astype(np.int64)
    return r


def dilate(mask, r):
    """Binary dilation by a (2r+1)^2 box (numpy only)."""
    out = mask.copy()
    if not mask.any():
        return out
    rows, cols = mask.shape
    ys, xs = np.nonzero(mask)
    for y, x in zip(ys, xs):
        out[max(0, y - r):min(rows, y + r + 1), max(0, x - r):min(cols, x + r + 1)] = True
    return out


def decision_stable_pixels(depth_u16, cam, idx32, idx64, max_radius=30):
    """Pixels whose normal computation takes the same discrete decisions in
    float and in double: same interval radius, and no pixel of its window
    (radius <= max_radius) changes validity between the two precisions."""
    r32 = radius_image(depth_u16, cam, np.float32)
    r64 = radius_image(depth_u16, cam, np.float64)
    bad_valid = (idx32 >= 0) != (idx64 >= 0)
    unstable = dilate(bad_valid, max_radius + 1) | (r32 != r64)
    return ~unstable, float(np.mean(r32 != r64)), int(bad_valid.sum())


def match_by_pixel(idx_a, idx_b, mask=None):
    """Point index pairs (a, b) of pixels valid in both index images."""
    m = (idx_a >= 0) & (idx_b >= 0)
    if mask is not None:
        m &= mask
    return idx_a[m], idx_b[m]
