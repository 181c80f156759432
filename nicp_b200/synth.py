"""Seeded synthetic NICP inputs: procedural rooms, camera poses and workloads.

Frames are rendered by libnicp_synth.so (include/nicp_synth.h).  Poses are
camera-to-world 4x4 matrices (x right, y down, z forward); the ground-truth
alignment of a (reference, current) pair is inv(pose_ref) @ pose_cur, the
transform that maps current-frame points into the reference frame -- what
AlignerProjective::T() estimates.
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(HERE, "libnicp_synth.so")

ROOM, FAR_ROOM = 0, 1
SIGMA_COEF = 0.0015   # depth noise sigma = 0.0015 * z^2 metres
DROP_PROB = 0.02      # fraction of zeroed pixels


class Scene(C.Structure):
    _fields_ = [("room_min", C.c_double * 3), ("room_max", C.c_double * 3), ("num_spheres", C.c_int),
                ("spheres", (C.c_double * 4) * 16), ("num_boxes", C.c_int), ("boxes", (C.c_double * 6) * 16)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError("libnicp_synth.so is missing: run `python -m nicp_b200.build`")
        lib = C.CDLL(SYNTH_PATH)
        lib.nicp_synth_scene_make.restype = C.c_int
        lib.nicp_synth_scene_make.argtypes = [C.c_uint64, C.c_int, C.POINTER(Scene)]
        lib.nicp_synth_render.restype = C.c_int
        lib.nicp_synth_render.argtypes = [C.POINTER(Scene), C.POINTER(C.c_double), C.c_float, C.c_float, C.c_float,
                                          C.c_float, C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_double,
                                          C.POINTER(C.c_uint16)]
        _lib = lib
    return _lib


def make_scene(seed, kind=ROOM):
    s = Scene()
    if _load().nicp_synth_scene_make(seed, kind, C.byref(s)) != 0:
        raise RuntimeError("scene generation failed")
    return s


def render(scene, pose, fx, fy, cx, cy, rows, cols, noise_seed, sigma_coef=SIGMA_COEF, drop_prob=DROP_PROB):
    """Renders a rows x cols uint16 depth image (millimetres)."""
    pose = np.ascontiguousarray(pose, dtype=np.float64).reshape(4, 4)
    out = np.zeros((rows, cols), dtype=np.uint16)
    n = _load().nicp_synth_render(C.byref(scene), pose.ctypes.data_as(C.POINTER(C.c_double)), fx, fy, cx, cy, rows,
                                  cols, noise_seed, sigma_coef, drop_prob, out.ctypes.data_as(C.POINTER(C.c_uint16)))
    if n < 0:
        raise RuntimeError("render failed")
    return out


# ------------------------------------------------------------------ SE(3) helpers
def rot(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = math.cos(angle), math.sin(angle)
    C1 = 1 - c
    return np.array([[c + x * x * C1, x * y * C1 - z * s, x * z * C1 + y * s],
                     [y * x * C1 + z * s, c + y * y * C1, y * z * C1 - x * s],
                     [z * x * C1 - y * s, z * y * C1 + x * s, c + z * z * C1]])


def make_T(R=None, t=None):
    T = np.eye(4)
    if R is not None:
        T[:3, :3] = R
    if t is not None:
        T[:3, 3] = t
    return T


def ypr(yaw, pitch, roll):
    return rot([0, 1, 0], yaw) @ rot([1, 0, 0], pitch) @ rot([0, 0, 1], roll)


def random_offset(rng, deg_lo, deg_hi, m_lo, m_hi):
    """A rigid offset with a random-axis rotation of deg in [deg_lo, deg_hi]
    and a random-direction translation of length in [m_lo, m_hi]."""
    ax = rng.normal(size=3)
    ang = math.radians(rng.uniform(deg_lo, deg_hi))
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    return make_T(rot(ax, ang), d * rng.uniform(m_lo, m_hi))


def rel(pose_ref, pose_cur):
    """Ground-truth T (current -> reference)."""
    return np.linalg.inv(pose_ref) @ pose_cur


def rot_angle(R):
    """Rotation angle of R: atan2(|axis term|, trace term), accurate at small
    angles (acos((tr - 1) / 2) loses half the digits there, and clips to 0
    when a float32 rotation's rounding puts the trace above 3)."""
    R = np.asarray(R, float)[:3, :3]
    s = math.sqrt((R[2, 1] - R[1, 2]) ** 2 + (R[0, 2] - R[2, 0]) ** 2 + (R[1, 0] - R[0, 1]) ** 2)
    return math.atan2(s, np.trace(R) - 1.0)


def pose_error(T_est, T_ref):
    """(rotation error in rad, translation error in m) of T_est vs T_ref."""
    D = np.linalg.inv(T_ref) @ T_est
    return rot_angle(D), float(np.linalg.norm(D[:3, 3]))


# ------------------------------------------------------------------ cameras / workloads
CAMERAS = {
    # name: (rows, cols, fx, fy, cx, cy)
    "160x120": (120, 160, 131.25, 131.25, 79.5, 59.5),
    "320x240": (240, 320, 262.5, 262.5, 159.5, 119.5),
    "640x480": (480, 640, 525.0, 525.0, 319.5, 239.5),
    "1280x720": (720, 1280, 1050.0, 1050.0, 639.5, 359.5),
}


def base_pose(rng, kind=ROOM):
    if kind == FAR_ROOM:
        return make_T(ypr(rng.uniform(-0.1, 0.1), rng.uniform(-0.05, 0.05), 0.0),
                      [rng.uniform(-0.3, 0.3), rng.uniform(-0.2, 0.2), 0.0])
    return make_T(ypr(rng.uniform(-0.15, 0.15), rng.uniform(-0.08, 0.08), rng.uniform(-0.05, 0.05)),
                  [rng.uniform(-0.2, 0.2), rng.uniform(-0.15, 0.15), -1.8 + rng.uniform(-0.1, 0.1)])


def trajectory(seed, n_frames=200, kind=ROOM, period=None):
    """A smooth periodic camera path through the room, one loop every
    `period` frames (default n_frames): with a period of 200 or more the
    per-frame steps stay below 1.5 degrees and 2 cm."""
    period = period or n_frames
    rng = np.random.default_rng(seed)
    P0 = base_pose(rng, kind)
    ph = rng.uniform(0, 2 * math.pi, size=6)
    poses = []
    for k in range(n_frames):
        w = 2 * math.pi * k / period
        yaw = math.radians(15) * math.sin(w + ph[0])
        pitch = math.radians(6) * math.sin(2 * w + ph[1])
        roll = math.radians(4) * math.sin(w + ph[2])
        t = np.array([0.25 * math.sin(w + ph[3]), 0.10 * math.sin(2 * w + ph[4]), 0.30 * math.sin(w + ph[5])])
        poses.append(P0 @ make_T(ypr(yaw, pitch, roll), t))
    return poses


def camera_dict(name, min_distance=0.01, max_distance=6.0):
    rows, cols, fx, fy, cx, cy = CAMERAS[name]
    return dict(rows=rows, cols=cols, fx=fx, fy=fy, cx=cx, cy=cy, min_distance=min_distance,
                max_distance=max_distance)


def render_pair(seed, cam_name="320x240", deg=2.0, meters=0.03, deg_hi=None, m_hi=None, kind=ROOM,
                sigma_coef=SIGMA_COEF, drop_prob=DROP_PROB):
    """A frame pair of one seeded scene: the current frame is rendered from the
    reference pose perturbed by a random rigid offset.  Returns
    (depth_ref, depth_cur, T_gt (current -> reference), camera dict)."""
    rng = np.random.default_rng(seed)
    scene = make_scene(seed, kind)
    P1 = base_pose(rng, kind)
    off = random_offset(rng, deg, deg if deg_hi is None else deg_hi, meters, meters if m_hi is None else m_hi)
    P2 = P1 @ off
    cam = camera_dict(cam_name, max_distance=(8.5 if kind == FAR_ROOM else 6.0))
    args = (cam["fx"], cam["fy"], cam["cx"], cam["cy"], cam["rows"], cam["cols"])
    d1 = render(scene, P1, *args, noise_seed=seed * 2 + 1, sigma_coef=sigma_coef, drop_prob=drop_prob)
    d2 = render(scene, P2, *args, noise_seed=seed * 2 + 2, sigma_coef=sigma_coef, drop_prob=drop_prob)
    return d1, d2, rel(P1, P2), cam


def render_sequence(seed, cam_name="640x480", n_frames=200, kind=ROOM, sigma_coef=SIGMA_COEF, drop_prob=DROP_PROB,
                    period=None):
    """Frames of the seeded smooth trajectory (one loop every `period`
    frames, default n_frames); returns (frames, poses, camera dict)."""
    scene = make_scene(seed, kind)
    poses = trajectory(seed, n_frames, kind, period)
    cam = camera_dict(cam_name)
    args = (cam["fx"], cam["fy"], cam["cx"], cam["cy"], cam["rows"], cam["cols"])
    frames = [render(scene, P, *args, noise_seed=seed * 100003 + k, sigma_coef=sigma_coef, drop_prob=drop_prob)
              for k, P in enumerate(poses)]
    return frames, poses, cam
