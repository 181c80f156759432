"""The committed golden fixture (tests/golden/pair_320x240.npz, written by
tests/golden/make_golden.py): the 320x240 plain-NICP pair with the oracle's
index image, point checksum, FP64 normal sample, correspondence checksum,
FP64 H/b and both pipelines' final poses.

CPU: the oracle still reproduces the fixture (regression guard of the
checker itself).  GPU: the CUDA path reproduces the index image and points
bit for bit, the FP64 normals within 1e-5 rad, and a final pose within
1e-5 rad / 0.05 mm of the FP64 pipeline's."""
import hashlib
import os

import numpy as np
import pytest

from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import angle_between, cams, converter, gpu_cloud

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pair_320x240.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def gold():
    g = np.load(GOLD)
    fx, fy, cx, cy, rows, cols = g["camera"]
    cam = dict(rows=int(rows), cols=int(cols), fx=float(fx), fy=float(fy), cx=float(cx), cy=float(cy),
               min_distance=0.01, max_distance=6.0)
    return g, cam


def test_oracle_reproduces_fixture(gold):
    g, cam = gold
    pc, oc = cams(cam)
    r32, i32 = O.build_cloud(O.REF32, g["depth_ref"], oc)
    assert np.array_equal(i32, g["index_ref"])
    assert sha(r32.get("points").astype(np.float32).reshape(-1, 4)) == str(g["points_ref_sha256"])
    r64, i64 = O.build_cloud(O.F64, g["depth_ref"], oc)
    rows, cols = g["sample_pixels"].T
    k = i64[rows, cols]
    got = np.concatenate([r64.get("normals").reshape(-1, 4)[k, :3], r64.get("curvature")[k, None]], axis=1)
    assert np.allclose(got, g["sample_normals_f64"], rtol=0, atol=1e-12)
    c32, _ = O.build_cloud(O.REF32, g["depth_cur"], oc)
    Tgt = g["T_gt"]
    ri, _ = O.project(O.REF32, r32, oc, Tgt)
    ci, _ = O.project(O.REF32, c32, oc, np.eye(4))
    corr = O.correspond(O.REF32, r32, c32, ri, ci, np.linalg.inv(Tgt))
    assert len(corr) == int(g["n_corr_ref32"]) and sha(corr.astype(np.int32)) == str(g["corr_ref32_sha256"])
    T32 = O.align(O.REF32, r32, c32, oc)["T"]
    assert np.max(np.abs(T32 - g["T_ref32"])) < 1e-12


@pytest.mark.gpu
def test_gpu_matches_fixture(ctx, gold):
    g, cam = gold
    proj, conv = converter(cam, ctx)
    ref, idx = gpu_cloud(ctx, conv, g["depth_ref"])
    assert np.array_equal(idx, g["index_ref"])
    d = ref.download()
    assert len(d["points"]) == int(g["n_points_ref"])
    assert sha(d["points"].astype(np.float32)) == str(g["points_ref_sha256"])
    rows, cols = g["sample_pixels"].T
    k = idx[rows, cols]
    ang = angle_between(d["normals"][k, :3].astype(np.float64), g["sample_normals_f64"][:, :3])
    assert np.max(ang) < 1e-5
    assert np.max(np.abs(d["curvature"][k] - g["sample_normals_f64"][:, 3])) < 1e-5
    cur, _ = gpu_cloud(ctx, conv, g["depth_cur"], keep_index=False)
    al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
    al.setReferenceCloud(ref)
    al.setCurrentCloud(cur)
    al.align()
    # Within 1e-5 rad / 0.05 mm of the FP64 pipeline, which starts from the
    # same float depth image (the REF32 pipeline, the reference's own float
    # arithmetic, ends ~1e-3 rad away: its FP32 integral moments).
    er, et = synth.pose_error(al.T(), g["T_f64"])
    e32, t32 = synth.pose_error(g["T_ref32"], g["T_f64"])
    print("golden pair: GPU vs FP64 %.3g rad %.3g m; REF32 vs FP64 %.3g rad %.3g m" % (er, et, e32, t32))
    assert er < 1e-5 and et < 5e-5, (er, et)
