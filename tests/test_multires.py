"""Coarse input (DepthImage_scale, imageutils.cpp:6-37), as the reference's
aligner apps run it for an image scale > 1 (nicp_aligner.cpp:152-163: the
depth image scaled, the camera matrix times 1/scale).

CPU: the oracle's block means and variance rejection against a numpy
evaluation of the same rule.  GPU: the scaled image equals the oracle's bit
for bit (u16 and float inputs, steps 1, 2, 3, 4), and a half-resolution
cloud built from it matches the oracle's (index image and points bit-exact)
and aligns like the FP64 oracle pipeline at that resolution."""
import numpy as np
import pytest

from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import cams, projector


def _numpy_scale(f, step, cov):
    rows, cols = f.shape[0] // step, f.shape[1] // step
    out = np.zeros((rows, cols), np.float32)
    for r in range(rows):
        for c in range(cols):
            b = f[r * step:(r + 1) * step, c * step:(c + 1) * step].astype(np.float64)
            np_ = int((b > 0).sum())
            if np_:
                mu = b.sum() / np_
                if (b * b).sum() / np_ - mu * mu <= cov:
                    out[r, c] = mu
    return out


def test_oracle_scale_rule():
    d1, _, _, cam = synth.render_pair(8, "160x120")
    f = O.convert_u16(d1)
    f[10:14, 20:24] = 0.0        # an empty block
    f[30, 40] = 5.0              # a block with a jump: variance rejection
    for step in (2, 4):
        o = O.depth_scale(f, step)
        ref = _numpy_scale(f, step, 0.01)
        assert o.shape == ref.shape
        # float vs double sums: equal up to rounding, same rejections
        assert np.array_equal(o > 0, ref > 0)
        assert np.max(np.abs(o - ref)) < 1e-5
    assert O.depth_scale(f, 2)[5, 10] == 0.0 and O.depth_scale(f, 2)[15, 20] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("step", [1, 2, 3, 4])
def test_scale_bitexact(ctx, step):
    d1, _, _, cam = synth.render_pair(9, "640x480")
    f = O.convert_u16(d1)
    want = O.depth_scale(f, step)
    assert np.array_equal(api.DepthImage_scale(d1, step, ctx=ctx), want)
    assert np.array_equal(api.DepthImage_scale(f, step, ctx=ctx), want)


@pytest.mark.gpu
def test_half_resolution_pipeline(ctx):
    d1, d2, Tgt, cam = synth.render_pair(12, "640x480")
    s1 = api.DepthImage_scale(d1, 2, ctx=ctx)
    s2 = api.DepthImage_scale(d2, 2, ctx=ctx)
    # nicp_aligner.cpp:155-163: the camera matrix times 1/imageScale (row 2
    # kept), the image size of the scaled depth
    half = dict(cam, rows=cam["rows"] // 2, cols=cam["cols"] // 2, fx=cam["fx"] * 0.5, fy=cam["fy"] * 0.5,
                cx=cam["cx"] * 0.5, cy=cam["cy"] * 0.5)
    proj = projector(half, ctx)
    conv = api.DepthImageConverterIntegralImage(proj, api.StatsCalculatorIntegralImage(),
                                                api.PointInformationMatrixCalculator(),
                                                api.NormalInformationMatrixCalculator())
    ref, cur = api.Cloud(ctx), api.Cloud(ctx)
    conv.compute(ref, s1, keep_index=True)
    idx = conv.indexImage()
    conv.compute(cur, s2)
    pc, oc = cams(half)
    o32, oidx = O.build_cloud_f32(O.REF32, s1, oc)
    assert np.array_equal(idx, oidx)
    assert np.array_equal(ref.download()["points"], o32.get("points").reshape(-1, 4).astype(np.float32))
    al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
    al.computeStatistics = False
    al.setReferenceCloud(ref)
    al.setCurrentCloud(cur)
    al.align()
    f1, _ = O.build_cloud_f32(O.F64, s1, oc)
    f2, _ = O.build_cloud_f32(O.F64, s2, oc)
    r = O.align(O.F64, f1, f2, oc)
    er, et = synth.pose_error(al.T(), r["T"])
    e32 = synth.pose_error(r["T"], Tgt)
    assert er < 1e-4 and et < 1e-4, (er, et, e32)
