"""Precision study at 1280x720, far range (fx = fy = 1050, depths 0.5-8 m;
maxDistance 8.5 so the far points stay in).

Variants: integral moments in FP32, compensated two-float or FP64; the
Linearizer's cross-block sum (the per-tile partials) in FP32 or FP64; the 6x6
LDLT is always FP64.  Per variant the table holds the normal angle and
curvature error against the FP64 oracle (pixels whose discrete decisions
agree), the H/b relative error against the FP64 oracle on identical clouds
and correspondences, the final pose error against the FP64 oracle pipeline,
and the device time of the cloud build and of the alignment.  The table is
written as JSON to $NICP_PRECISION_TABLE when that is set.

Gates: FP64 and two-float moments meet the 1e-5 rad normal gate; with FP64
moments and an FP64 cross-block sum, H/b are within 1e-5 relative and the
converged pose (30 outer iterations) within 1e-5 rad / 0.05 mm of the FP64
oracle.  At the reference's 10 outer iterations this far-range pair has not
converged yet (the oracle's own pose still differs from its 30-iteration
pose by more than the gate), so the two pipelines' last-bit differences
along the way are visible there; that figure is reported beside the gated
one.  The FP32 variants are reported, not gated.
"""
import json
import os

import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import (angle_between, cams, converter, decision_stable_pixels, float_T, gpu_cloud, match_by_pixel,
                     oracle_cloud_from_gpu, perturb)

pytestmark = pytest.mark.gpu

MOMENTS = [("fp64", L.NICP_MOMENTS_F64), ("twofloat", L.NICP_MOMENTS_TWOFLOAT), ("fp32", L.NICP_MOMENTS_F32)]
BUILD_KERNELS = ("unproject", "moments_bands", "moments_sweep", "stats_omega")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def far():
    d1, d2, Tgt, cam = synth.render_pair(41, "1280x720", kind=synth.FAR_ROOM)
    assert cam["max_distance"] >= 8.0
    pc, oc = cams(cam)
    ref, ridx = O.build_cloud(O.F64, d1, oc)
    cur, _ = O.build_cloud(O.F64, d2, oc)
    r = O.align(O.F64, ref, cur, oc)
    r30 = O.align(O.F64, ref, cur, oc, prm=O.align_params(outer_iterations=30))
    return dict(d1=d1, d2=d2, Tgt=Tgt, cam=cam, ref=ref, ridx=ridx, T=r["T"], T30=r30["T"])


def _build(ctx, conv, depth):
    gpu_cloud(ctx, conv, depth)  # first launches load the kernels: not timed
    ctx.set_profiling(True)
    c, idx = gpu_cloud(ctx, conv, depth)
    ms = sum(ctx.read_profile(k)[0] for k in BUILD_KERNELS)
    ctx.set_profiling(False)
    return c, idx, ms


def _row(ctx, far, mname, prec, cross_f32):
    cam = far["cam"]
    proj, conv = converter(cam, ctx, precision=prec)
    ref, ri, ms_ref = _build(ctx, conv, far["d1"])
    cur, _, ms_cur = _build(ctx, conv, far["d2"])
    row = {"moments": mname, "cross_block": "fp32" if cross_f32 else "fp64",
           "build_ms_per_frame": 0.5 * (ms_ref + ms_cur)}

    # normals and curvature against the FP64 oracle cloud
    f = far["ref"]
    stable, _, _ = decision_stable_pixels(far["d1"], cam, ri, far["ridx"])
    gi, fi = match_by_pixel(ri, far["ridx"], stable)
    g = ref.download()
    fn, lam, fk = f.get("normals")[fi, :3], f.get("eigenvalues")[fi], f.get("curvature")[fi]
    gn, gk = g["normals"][gi, :3].astype(np.float64), g["curvature"][gi].astype(np.float64)
    both = (np.abs(fn).sum(1) > 0) & (np.abs(gn).sum(1) > 0) & ((lam[:, 1] - lam[:, 0]) > 1e-3 * lam[:, 2])
    ang = angle_between(fn[both], gn[both])
    dk = np.abs(gk[both] - fk[both])
    row.update(normal_angle_max_rad=float(np.max(ang)), normal_angle_median_rad=float(np.median(ang)),
               curvature_abs_max=float(np.max(dk)), curvature_abs_median=float(np.median(dk)),
               compared_points=int(both.sum()))

    # H and b on identical inputs (this variant's clouds, correspondences at
    # the oracle's final pose moved by 1 deg / 2 cm, where b is far from 0)
    T = far["T"] @ perturb(7, 1.0, 0.02)
    proj.setTransform(np.eye(4))
    cur_idx, _ = proj.project(cur)
    proj.setTransform(float_T(T))
    ref_idx, _ = proj.project(ref)
    cf = api.CorrespondenceFinderProjective(ctx)
    cf.setReferenceIndexImage(ref_idx)
    cf.setCurrentIndexImage(cur_idx)
    Tinv = np.linalg.inv(float_T(T)).astype(np.float32)
    pairs = cf.compute(ref, cur, Tinv)
    lin = api.Linearizer(ctx)
    lin.crossBlockF32 = cross_f32
    lin.setT(Tinv)
    lin.update(ref, cur, pairs)
    oref = oracle_cloud_from_gpu(O.F64, ref.download())
    ocur = oracle_cloud_from_gpu(O.F64, cur.download())
    H, b, err, inl = O.linearize(O.F64, oref, ocur, pairs, Tinv.astype(np.float64))
    row.update(H_rel=_rel(lin.H(), H), b_rel=_rel(lin.b(), b), correspondences=int(len(pairs)))

    # the whole pipeline against the FP64 oracle pipeline (10 outer
    # iterations, the reference default, and 30)
    proj.setTransform(np.eye(4))
    for outer, key in ((10, ""), (30, "_30")):
        lin2 = api.Linearizer(ctx)
        lin2.crossBlockF32 = cross_f32
        al = api.AlignerProjective(proj, lin2, api.CorrespondenceFinderProjective(ctx), ctx)
        al.computeStatistics = False
        al.setOuterIterations(outer)
        al.setReferenceCloud(ref)
        al.setCurrentCloud(cur)
        al.align()
        ctx.set_profiling(True)
        al.align()
        align_ms = sum(ctx.read_profile(k)[0] for k in L.KERNELS)
        ctx.set_profiling(False)
        er, et = synth.pose_error(al.T(), far["T" + ("30" if key else "")])
        row.update({"pose_err_rad" + key: float(er), "pose_err_m" + key: float(et), "align_ms" + key: align_ms})
    return row


def test_precision_study(ctx, far):
    rows = []
    for mname, prec in MOMENTS:
        for cross_f32 in (False, True):
            rows.append(_row(ctx, far, mname, prec, cross_f32))
    table = {"workload": "1280x720 far-range pair (seed 41), fx=fy=1050, maxDistance 8.5, 10 outer x 1 inner",
             "truth_vs_f64_oracle": dict(zip(("rad", "m"), map(float, synth.pose_error(far["T"], far["Tgt"])))),
             "f64_oracle_10_vs_30_iterations": dict(zip(("rad", "m"),
                                                        map(float, synth.pose_error(far["T"], far["T30"])))),
             "rows": rows}
    out = os.environ.get("NICP_PRECISION_TABLE")
    if out:
        with open(out, "w") as fh:
            json.dump(table, fh, indent=1)
    for r in rows:
        print(json.dumps(r))
    by = {(r["moments"], r["cross_block"]): r for r in rows}
    for m in ("fp64", "twofloat"):
        assert by[(m, "fp64")]["normal_angle_max_rad"] < 1e-5, by[(m, "fp64")]
    best = by[("fp64", "fp64")]
    assert best["H_rel"] < 1e-5 and best["b_rel"] < 1e-5, best
    # the reference's 10 outer iterations and a converged 30
    assert best["pose_err_rad"] < 1e-5 and best["pose_err_m"] < 5e-5, best
    assert best["pose_err_rad_30"] < 1e-5 and best["pose_err_m_30"] < 5e-5, best
