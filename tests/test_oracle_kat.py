"""Known-answer tests of the CPU oracle (no GPU).  The reference ships no
tests or golden vectors, so the restatement is pinned here against
independent numpy computations and analytic answers."""
import math

import numpy as np
import pytest

from nicp_b200 import synth
from oracle import oracle as O


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _spd(rng, scale=1.0):
    A = rng.normal(size=(3, 3)) * scale
    return A @ A.T


@pytest.mark.parametrize("mode", [O.F64, O.REF32])
def test_eig3_matches_numpy(mode):
    rng = np.random.default_rng(1)
    tol = 1e-12 if mode == O.F64 else 2e-5
    for k in range(300):
        S = _spd(rng, 10 ** rng.uniform(-3, 1))
        if k % 3 == 1:  # near-planar covariance, as on flat surfaces
            w, V = np.linalg.eigh(S)
            S = V @ np.diag([w[2] * 1e-6, w[1], w[2]]) @ V.T
        A6 = [S[0, 0], S[0, 1], S[0, 2], S[1, 1], S[1, 2], S[2, 2]]
        lam, U = O.eig3(mode, A6)
        w, V = np.linalg.eigh(S)
        assert np.allclose(lam, w, atol=tol * max(1.0, w[2]), rtol=0), (lam, w)
        assert np.allclose(U.T @ U, np.eye(3), atol=10 * tol)
        if w[1] - w[0] > 1e-3 * w[2]:
            assert abs(abs(U[:, 0] @ V[:, 0]) - 1) < 10 * tol


def test_eig3_degenerate():
    """Repeated eigenvalues.  The trigonometric roots of the cubic resolve a
    double root only to about sqrt(eps) * lambda_max (acos is ill-conditioned
    at +-1); the basis stays orthonormal and S U = U diag(lambda) holds to
    the same order."""
    for S in [np.eye(3), np.zeros((3, 3)), np.diag([2.0, 2.0, 5.0]), np.outer([1, 2, 3], [1, 2, 3]) * 1.0]:
        lam, U = O.eig3(O.F64, [S[0, 0], S[0, 1], S[0, 2], S[1, 1], S[1, 2], S[2, 2]])
        tol = 2e-8 * max(1.0, np.max(np.abs(S)))
        assert np.allclose(np.sort(lam), np.linalg.eigvalsh(S), atol=tol)
        assert np.allclose(U.T @ U, np.eye(3), atol=1e-12)
        assert np.allclose(S @ U, U @ np.diag(lam), atol=tol)


@pytest.mark.parametrize("mode", [O.F64, O.REF32])
def test_ldlt_solve(mode):
    rng = np.random.default_rng(2)
    for _ in range(50):
        A = rng.normal(size=(6, 6))
        H = A @ A.T + 1e3 * np.eye(6) * rng.uniform(0.01, 10)
        b = rng.normal(size=6)
        x = O.ldlt_solve(mode, H, b)
        ref = np.linalg.solve(H, b)
        assert np.allclose(x, ref, rtol=1e-10 if mode == O.F64 else 1e-4, atol=1e-12)


@pytest.mark.parametrize("mode", [O.F64, O.REF32])
def test_se3_round_trip(mode):
    rng = np.random.default_rng(3)
    tol = 1e-12 if mode == O.F64 else 1e-6
    for _ in range(100):
        T = synth.random_offset(rng, 0.0, 170.0, 0.0, 3.0)
        x = O.t2v(mode, T)
        T2 = O.v2t(mode, x)
        assert np.allclose(T2, T, atol=tol)
        assert np.allclose(O.iso_inverse(mode, T) @ T, np.eye(4), atol=tol)
        # the vector part belongs to a quaternion with w >= 0
        assert np.linalg.norm(x[3:]) <= 1 + tol


def test_integral_region_window_rule():
    """getRegion sums the box cols (c-r-1, c+r-1], rows (r-r-1, r+r-1] after
    clamping each bound (pointintegralimage.cpp:53-66)."""
    rng = np.random.default_rng(4)
    rows, cols = 23, 31
    idx = -np.ones((rows, cols), np.int32)
    valid = rng.uniform(size=(rows, cols)) < 0.8
    idx[valid] = np.arange(valid.sum())
    pts = np.zeros((valid.sum(), 4))
    pts[:, :3] = rng.normal(size=(valid.sum(), 3))
    pts[:, 3] = 1
    cl = O.Cloud.from_arrays(O.F64, pts, np.zeros_like(pts), np.zeros(len(pts)))
    for _ in range(200):
        x0, x1 = sorted(rng.integers(-5, cols + 5, size=2))
        y0, y1 = sorted(rng.integers(-5, rows + 5, size=2))
        got = O.integral_region(O.F64, cl, idx, x0, x1, y0, y1)
        cm = lambda v: min(max(v - 1, 0), cols - 1)
        rm = lambda v: min(max(v - 1, 0), rows - 1)
        xa, xb, ya, yb = cm(x0), cm(x1), rm(y0), rm(y1)
        sub = idx[ya + 1:yb + 1, xa + 1:xb + 1]
        sel = pts[sub[sub >= 0]]
        p = sel[:, :3]
        exp = [len(sel), *p.sum(0), (p[:, 0] ** 2).sum(), (p[:, 0] * p[:, 1]).sum(), (p[:, 0] * p[:, 2]).sum(),
               (p[:, 1] ** 2).sum(), (p[:, 1] * p[:, 2]).sum(), (p[:, 2] ** 2).sum()]
        assert np.allclose(got, exp, atol=1e-9), (x0, x1, y0, y1)


def _plane_depth(rows, cols, fx, fy, cx, cy, n, c, scale=1e-4):
    u, v = np.meshgrid(np.arange(cols), np.arange(rows))
    dirs = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u, float)], -1)
    z = c / (dirs @ n)
    return np.clip(np.round(z / scale), 0, 65535).astype(np.uint16)


def test_unprojection_analytic():
    cam = synth.camera_dict("160x120")
    d = np.full((cam["rows"], cam["cols"]), 2000, np.uint16)
    d[5, 7] = 0
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    cl, idx = O.build_cloud(O.F64, d, oc)
    assert idx[5, 7] == -1 and idx[0, 0] == 0 and idx[5, 8] == 5 * cam["cols"] + 7
    P = cl.get("points")
    z = np.float64(np.float32(0.001) * np.float32(2000))  # the float DepthImage, promoted
    r, c = 10, 20
    k = idx[r, c]
    assert np.allclose(P[k, :3], [(c - cam["cx"]) / cam["fx"] * z, (r - cam["cy"]) / cam["fy"] * z, z], atol=1e-12)


def test_stats_match_brute_force_windows():
    """Normals, curvature and information matrices of the F64 oracle equal a
    brute-force numpy evaluation of the reference's window rule (interval
    radius, clamps, min points), covariance and eigendecomposition."""
    d1, _, _, cam = synth.render_pair(9, "320x240")
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    cl, idx = O.build_cloud(O.F64, d1, oc)
    P, N, K = cl.get("points"), cl.get("normals"), cl.get("curvature")
    OP = cl.get("omega_p").reshape(-1, 3, 3)
    rows, cols = idx.shape
    rng = np.random.default_rng(5)
    checked = 0
    for _ in range(400):
        r, c = int(rng.integers(rows)), int(rng.integers(cols))
        k = idx[r, c]
        if k < 0:
            continue
        z = np.float64(np.float32(0.001) * np.float32(int(d1[r, c])))  # the float DepthImage, promoted
        R = np.float64(np.float32(0.1))
        rad = int(max(cam["fx"] * R * (1 / z), cam["fy"] * R * (1 / z)))
        if rad < 10:
            assert not N[k].any()
            continue
        rad = min(rad, 30)
        cm = lambda v: min(max(v - 1, 0), cols - 1)
        rm = lambda v: min(max(v - 1, 0), rows - 1)
        sub = idx[rm(r - rad) + 1:rm(r + rad) + 1, cm(c - rad) + 1:cm(c + rad) + 1]
        sel = P[sub[sub >= 0], :3]
        if len(sel) < 50:
            assert not N[k].any()
            continue
        C = np.cov(sel.T, bias=True)
        w, V = np.linalg.eigh(C)
        w[0] = max(w[0], 0)
        kap = w[0] / (w.sum() + 1e-9)
        assert abs(kap - K[k]) < 1e-9
        if kap < 0.02:
            n = V[:, 0] * (-1 if V[:, 0] @ P[k, :3] > 0 else 1)
            if w[1] - w[0] > 1e-3 * w[2]:
                assert np.allclose(N[k, :3], n, atol=1e-7), (N[k], n)
                exp = V @ np.diag([1000, 0.001, 0.001]) @ V.T
                assert np.allclose(OP[k], exp, atol=1e-5)
            checked += 1
        else:
            assert not N[k].any()
    assert checked > 50


def test_plane_normals_analytic():
    """A noise-free tilted plane: every normal is the plane normal, curvature ~0."""
    cam = synth.camera_dict("320x240")
    n = np.array([0.2, -0.3, 1.0])
    n /= np.linalg.norm(n)
    d = _plane_depth(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"], n, 1.5)
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    prm = O.cloud_params(depth_scale=1e-4)
    cl, idx = O.build_cloud(O.F64, d, oc, prm)
    N = cl.get("normals")[:, :3]
    has = np.abs(N).sum(1) > 0
    assert has.mean() > 0.8
    # normals face the camera: n . p < 0
    ang = np.arccos(np.clip(np.abs(N[has] @ n), 0, 1))
    assert np.max(ang) < 2e-3  # 0.1 mm depth quantization
    assert np.max(cl.get("curvature")[has]) < 1e-4


def test_zbuffer_ties_lowest_index():
    cam = dict(rows=8, cols=8, fx=4.0, fy=4.0, cx=3.5, cy=3.5)
    pts = np.array([[0, 0, 2, 1], [0, 0, 2, 1], [0, 0, 1.5, 1], [0, 0, 1.5, 1]], float)
    cl = O.Cloud.from_arrays(O.REF32, pts, np.zeros((4, 4)), np.zeros(4))
    oc = O.camera(8, 8, 4.0, 4.0, 3.5, 3.5)
    ii, dd = O.project(O.REF32, cl, oc, np.eye(4))
    assert ii[4, 4] == 2 and dd[4, 4] == np.float32(1.5)
    assert (ii >= 0).sum() == 1


@pytest.fixture(scope="module")
def pair640():
    d1, d2, Tgt, cam = synth.render_pair(13, "640x480", sigma_coef=0.0, drop_prob=0.0)
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    ref, ri = O.build_cloud(O.F64, d1, oc)
    cur, ci = O.build_cloud(O.F64, d2, oc)
    return dict(ref=ref, cur=cur, Tgt=Tgt, oc=oc, ri=ri, ci=ci)


def test_identity_alignment(pair640):
    """A cloud aligned with itself: H symmetric PSD, b ~ 0, T = I."""
    p = pair640
    I = np.eye(4)
    ci, _ = O.project(O.F64, p["ref"], p["oc"], I)
    pairs = O.correspond(O.F64, p["ref"], p["ref"], ci, ci, I)
    H, b, err, inl = O.linearize(O.F64, p["ref"], p["ref"], pairs, I)
    assert np.allclose(H, H.T, rtol=1e-9, atol=1e-6)
    assert np.min(np.linalg.eigvalsh(H)) > -1e-6 * np.max(np.abs(H))
    assert np.linalg.norm(b) < 1e-6 * np.linalg.norm(H)
    r = O.align(O.F64, p["ref"], p["ref"], p["oc"])
    assert np.allclose(r["T"], I, atol=1e-12)


def test_known_transform_recovered(pair640):
    """Noise-free 640x480 pair, 2 deg + 3 cm: recovered within 1e-3 rad / 3 mm."""
    p = pair640
    r = O.align(O.F64, p["ref"], p["cur"], p["oc"])
    er, et = synth.pose_error(r["T"], p["Tgt"])
    assert er < 1e-3 and et < 3e-3, (er, et)


def test_thread_partition_drops(pair640):
    """With T threads the reference skips the last rows % T image rows
    (correspondencefinderprojective.cpp:41,50-53) and the last K % T
    correspondences (linearizer.cpp:36,40-43)."""
    p = pair640
    ref = O.Cloud.from_arrays(O.REF32, p["ref"].get("points"), p["ref"].get("normals"), p["ref"].get("curvature"),
                              p["ref"].get("omega_p"), p["ref"].get("omega_n"))
    cur = O.Cloud.from_arrays(O.REF32, p["cur"].get("points"), p["cur"].get("normals"), p["cur"].get("curvature"),
                              p["cur"].get("omega_p"), p["cur"].get("omega_n"))
    ci, _ = O.project(O.REF32, cur, p["oc"], np.eye(4))
    ri, _ = O.project(O.REF32, ref, p["oc"], p["Tgt"])
    T = np.linalg.inv(p["Tgt"])
    full = O.correspond(O.REF32, ref, cur, ri, ci, T, O.align_params(threads=1))
    rows, cols = ri.shape
    # row of every correspondence in the full (row-major) list
    flat = ri.reshape(-1)
    row_of = {}
    for q in np.nonzero(flat >= 0)[0]:
        row_of[int(flat[q])] = int(q) // cols
    for th in (7, 13):
        got = O.correspond(O.REF32, ref, cur, ri, ci, T, O.align_params(threads=th))
        keep = [i for i, (a, b) in enumerate(full) if row_of[int(a)] < (rows // th) * th]
        assert np.array_equal(got, full[keep])
        Kk = (len(got) // th) * th
        H, b, e, n = O.linearize(O.REF32, ref, cur, got, T, O.align_params(threads=th))
        Hd, bd, ed, nd = O.linearize(O.REF32, ref, cur, got[:Kk], T, O.align_params(threads=1))
        assert n == nd == Kk
        # the reference's float partial sums depend on T: over ~1e5 terms the
        # 7- and 13-thread H differ from the sequential one by ~1e-3 relative
        # (which is why the CUDA path accumulates in FP64)
        Hf, bf, ef, nf = O.linearize(O.F64, p["ref"], p["cur"], got[:Kk], T)
        rel = np.linalg.norm(H - Hf) / np.linalg.norm(Hf)
        rel1 = np.linalg.norm(Hd - Hf) / np.linalg.norm(Hf)
        assert rel < 1e-2 and rel1 < 1e-2, (rel, rel1)


def test_unprojection_gaussian_analytic():
    """Gaussian3f of unProject (pinholepointprojector.cpp:93-134): with
    K^-1 [[z,0,c],[0,z,r],[0,0,1]] = [[z/f,0,(c-cx)/f],[0,z/f,(r-cy)/f],[0,0,1]]
    the covariance is that matrix times diag(3, 3, a z^2/(f B + a z)) times
    its transpose; the mean is the point."""
    cam = synth.camera_dict("160x120")
    d = np.full((cam["rows"], cam["cols"]), 2500, np.uint16)
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    cl, idx = O.build_cloud(O.F64, d, oc)
    cov = cl.get("gaussian_cov").reshape(-1, 3, 3)
    mean = cl.get("gaussian_mean").reshape(-1, 3)
    z = np.float64(np.float32(0.001) * np.float32(2500))  # the float DepthImage, promoted
    f, B, a = cam["fx"], 0.075, np.float64(np.float32(0.1))
    for r, c in [(0, 0), (37, 101), (119, 159)]:
        k = idx[r, c]
        J = np.array([[z / f, 0, (c - cam["cx"]) / f], [0, z / f, (r - cam["cy"]) / f], [0, 0, 1.0]])
        zv = a * z * z / (f * np.float64(np.float32(B)) + z * a)
        exp = J @ np.diag([3.0, 3.0, zv]) @ J.T
        assert np.allclose(cov[k], exp, rtol=1e-9, atol=1e-15), (r, c)
        assert np.array_equal(mean[k], cl.get("points").reshape(-1, 4)[k, :3])


def test_correspond_multi_matches_brute_force():
    """_computeMulti (correspondencefinderprojective.cpp:119-257) restated:
    for a sample of reference pixels, a plain-Python scan of the clamped
    window (row-major; gates: current normal present, normal angle, distance,
    curvature ratio; a later candidate replaces the kept one only if strictly
    closer and strictly better aligned) picks the current point the oracle
    lists; regions 0 0 give the single-pixel list."""
    d1, d2, Tgt, cam = synth.render_pair(13, "160x120")
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    ref, _ = O.build_cloud(O.F64, d1, oc)
    cur, _ = O.build_cloud(O.F64, d2, oc)
    ri, _ = O.project(O.F64, ref, oc, Tgt)
    ci, _ = O.project(O.F64, cur, oc, np.eye(4))
    T = np.linalg.inv(Tgt)
    R, Cw = 2, 1
    prm = O.align_params(row_search_region=R, col_search_region=Cw)
    pairs = O.correspond(O.F64, ref, cur, ri, ci, T, prm)
    assert len(pairs) > 1000
    got = {int(a): int(b) for a, b in pairs}
    P, N, K = ref.get("points"), ref.get("normals"), ref.get("curvature")
    cP, cN, cK = cur.get("points"), cur.get("normals"), cur.get("curvature")
    p0 = O.align_params()
    sq = np.float64(np.float32(p0.inlier_distance_threshold)) ** 2
    cos_t, flat = p0.inlier_normal_angular_threshold, np.float64(np.float32(p0.flat_curvature_threshold))
    thr = np.float64(np.float32(p0.inlier_curvature_ratio_threshold))
    rows, cols = ri.shape
    rng = np.random.default_rng(3)
    checked = 0
    cand = np.argwhere((ri >= 0) & (np.abs(N[np.maximum(ri, 0), :3]).sum(-1) > 0))
    for r, c in cand[rng.choice(len(cand), size=min(300, len(cand)), replace=False)]:
        r, c = int(r), int(c)
        a = ri[r, c]
        rp = T[:3, :3] @ P[a, :3] + T[:3, 3]
        rn = T[:3, :3] @ N[a, :3]
        kr = max(K[a], flat)
        best, bn, bd = -1, 0.0, 1e20
        for r2 in range(max(r - R, 0), min(r + R + 1, rows)):
            for c2 in range(max(c - Cw, 0), min(c + Cw + 1, cols)):
                b = ci[r2, c2]
                if b < 0 or not cN[b, :3].any():
                    continue
                nd = float(cN[b, :3] @ rn)
                if nd < cos_t:
                    continue
                d = float(np.sum((cP[b, :3] - rp) ** 2))
                if d > sq:
                    continue
                ratio = (kr + 1e-5) / (max(cK[b], flat) + 1e-5)
                if ratio < 1.0 / thr or ratio > thr:
                    continue
                if best == -1 or (d < bd and nd > bn):
                    best, bn, bd = b, nd, d
        assert got.get(int(a), -1) == best, (r, c)
        checked += 1
    assert checked > 100
    single = O.correspond(O.F64, ref, cur, ri, ci, T, O.align_params())
    zero = O.correspond(O.F64, ref, cur, ri, ci, T, O.align_params(row_search_region=0, col_search_region=0))
    assert np.array_equal(single, zero)


def test_pose_sensitivity_to_one_ulp_of_depth():
    """How well the FP64 pose of the config-1 pair (the golden pair: 320x240,
    2 deg + 3 cm, reference defaults, 10 outer x 1 inner) is determined by
    its input: moving every float depth of the reference's DepthImage by one
    ulp, up or down at random, moves the FP64 pipeline's pose by more than
    1e-5 rad -- discrete decisions (window radii, validity, gates, pixel
    rounding) flip and the unconverged loop carries the difference on.  A
    float pipeline cannot be held closer to FP64 than this on this pair, so
    the pose gate of this pair is quoted together with these figures."""
    d1, d2, _, cam = synth.render_pair(1, "320x240", deg=2.0, meters=0.03)
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    f1, f2 = O.convert_u16(d1), O.convert_u16(d2)
    a, _ = O.build_cloud_f32(O.F64, f1, oc)
    b, _ = O.build_cloud_f32(O.F64, f2, oc)
    T0 = O.align(O.F64, a, b, oc)["T"]
    # the u16 path starts from the same float image
    a16, _ = O.build_cloud(O.F64, d1, oc)
    b16, _ = O.build_cloud(O.F64, d2, oc)
    assert np.array_equal(O.align(O.F64, a16, b16, oc)["T"], T0)
    moves = []
    for seed in (1, 2, 3):
        rng = np.random.default_rng(seed)

        def ulp(f):
            up = rng.integers(0, 2, size=f.shape).astype(bool)
            g = np.where(up, np.nextafter(f, np.float32(np.inf)), np.nextafter(f, np.float32(-np.inf)))
            return np.where(f > 0, g, f).astype(np.float32)

        pa, _ = O.build_cloud_f32(O.F64, ulp(f1), oc)
        pb, _ = O.build_cloud_f32(O.F64, ulp(f2), oc)
        moves.append(synth.pose_error(O.align(O.F64, pa, pb, oc)["T"], T0))
    print("FP64 pose moved by one-ulp depth perturbations: %s" % ["%.2e rad %.2e m" % m for m in moves])
    assert max(m[0] for m in moves) > 1e-5


def test_zero_normal_test_is_a_threshold():
    """The gates' "squaredNorm() == 0" (correspondencefinderprojective.cpp:69)
    is decided on the GPU as |x|, |y|, |z| <= 2^-75: a float sum of
    non-negative squares is zero exactly when every square rounds to zero,
    and x * x rounds to zero exactly at |x| <= 2^-75 (2^-150 ties to 0).
    Checked here in float32 arithmetic on the edge values and on random
    vectors spanning the subnormal range, NaN and infinity included."""
    t = np.float32(2.0 ** -75)
    edge = np.array([0.0, -0.0, t, -t, np.nextafter(t, np.float32(1)), np.nextafter(t, np.float32(0)),
                     np.float32(1e-40), np.float32(2.6e-23), np.float32(2.7e-23), np.float32(1e-20), 1.0,
                     np.inf, -np.inf, np.nan], np.float32)
    g = np.array(np.meshgrid(edge, edge, edge)).reshape(3, -1).T
    rng = np.random.default_rng(7)
    r = (rng.standard_normal((200000, 3)) * np.float32(2.0) ** rng.integers(-160, 10, (200000, 3))).astype(np.float32)
    r[rng.random(200000) < 0.3, 0] = 0.0
    v = np.concatenate([g, r]).astype(np.float32)
    with np.errstate(over="ignore", under="ignore", invalid="ignore"):
        x, y, z = v[:, 0], v[:, 1], v[:, 2]
        sq = ((x * x + y * y) + z * z).astype(np.float32)  # float32 throughout
        assert sq.dtype == np.float32
        zero_by_sum = sq == np.float32(0)
        zero_by_thr = (np.abs(x) <= t) & (np.abs(y) <= t) & (np.abs(z) <= t)
    assert np.array_equal(zero_by_sum, zero_by_thr)
    assert zero_by_thr.sum() > 100 and (~zero_by_thr).sum() > 100
