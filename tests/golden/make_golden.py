"""Writes the golden fixture tests/golden/pair_320x240.npz.

The reference ships no test vectors for this path, so the fixture holds
what the oracle computes on the 320x240 plain-NICP workload (a seeded
procedural room; the second frame 2 degrees about a random axis and 3 cm
away; fx = fy = 262.5, cx = 159.5, cy = 119.5; reference defaults, 10 outer
x 1 inner):

  depth_ref, depth_cur   the two uint16 frames (millimetres)
  T_gt                   ground truth, current -> reference
  index_ref              REF32 index image of the reference frame
  points_ref_sha256      sha256 of the REF32 points (float32, n x 4)
  n_points_ref           their count
  sample_pixels          (row, col) of 2000 pixels whose normal computation
                         takes the same discrete decisions in float and double
  sample_normals_f64     FP64 oracle normals (xyz) and curvature there
  corr_ref32_sha256      sha256 of the REF32 correspondence list at T_gt
                         (int32 pairs), and n_corr_ref32 its length
  H_f64, b_f64           FP64 Linearizer H and b at T_gt on the FP64 clouds
  T_ref32, T_f64         final poses of the REF32 and FP64 pipelines

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from nicp_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

from helpers import cams, decision_stable_pixels  # noqa: E402

SEED = 1
OUT = os.path.join(HERE, "pair_320x240.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    d1, d2, Tgt, cam = synth.render_pair(SEED, "320x240", deg=2.0, meters=0.03)
    pc, oc = cams(cam)
    r32, i32 = O.build_cloud(O.REF32, d1, oc)
    c32, _ = O.build_cloud(O.REF32, d2, oc)
    r64, i64 = O.build_cloud(O.F64, d1, oc)
    c64, _ = O.build_cloud(O.F64, d2, oc)
    pts = r32.get("points").astype(np.float32).reshape(-1, 4)

    stable, _, _ = decision_stable_pixels(d1, cam, i32, i64)
    n64 = r64.get("normals").reshape(-1, 4)
    k64 = r64.get("curvature")
    lam = r64.get("eigenvalues").reshape(-1, 3)
    rows, cols = np.nonzero(stable & (i64 >= 0))
    k = i64[rows, cols]
    good = (np.abs(n64[k, :3]).sum(1) > 0) & ((lam[k, 1] - lam[k, 0]) > 1e-3 * lam[k, 2])
    rows, cols, k = rows[good], cols[good], k[good]
    pick = np.random.default_rng(SEED).choice(len(k), size=2000, replace=False)
    pick.sort()
    rows, cols, k = rows[pick], cols[pick], k[pick]
    sample = np.concatenate([n64[k, :3], k64[k, None]], axis=1)

    # correspondences and Linearizer at the ground truth
    _, _, Tinv = None, None, np.linalg.inv(Tgt)
    ref_idx32, _ = O.project(O.REF32, r32, oc, Tgt)
    cur_idx32, _ = O.project(O.REF32, c32, oc, np.eye(4))
    corr32 = O.correspond(O.REF32, r32, c32, ref_idx32, cur_idx32, Tinv)
    ref_idx64, _ = O.project(O.F64, r64, oc, Tgt)
    cur_idx64, _ = O.project(O.F64, c64, oc, np.eye(4))
    corr64 = O.correspond(O.F64, r64, c64, ref_idx64, cur_idx64, Tinv)
    H, b, _, _ = O.linearize(O.F64, r64, c64, corr64, Tinv)

    T32 = O.align(O.REF32, r32, c32, oc)["T"]
    T64 = O.align(O.F64, r64, c64, oc)["T"]
    np.savez_compressed(OUT, depth_ref=d1, depth_cur=d2, T_gt=Tgt, index_ref=i32.astype(np.int32),
                        points_ref_sha256=sha(pts), n_points_ref=len(pts),
                        sample_pixels=np.stack([rows, cols], 1).astype(np.int32), sample_normals_f64=sample,
                        corr_ref32_sha256=sha(corr32.astype(np.int32)), n_corr_ref32=len(corr32),
                        H_f64=H, b_f64=b, T_ref32=T32, T_f64=T64,
                        camera=np.array([cam["fx"], cam["fy"], cam["cx"], cam["cy"], cam["rows"], cam["cols"]]))
    print("wrote", OUT, os.path.getsize(OUT), "bytes;", len(pts), "points,", len(corr32), "correspondences")


if __name__ == "__main__":
    main()
