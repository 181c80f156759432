"""Frame-to-scene fusion: Cloud::add (cloud.cpp:163-189) and Merger::merge
(merger.cpp:15-109), the CUDA path against the REF32 oracle.

CPU: the oracle's merge of a cloud with an exact copy of itself removes
every copy point and halves every covariance (information adds up).
GPU: on a two-frame scene (frame 0 + frame 1 added with the true relative
pose, merged in frame 1's view) and on the self-copy case, the surviving
points, their fused Gaussians and the number of removed points equal the
REF32 oracle bit for bit (same projection, same index-ordered information
sums, single-rounded float steps)."""
import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import cams, converter


def test_oracle_merge_of_a_copy():
    d1, _, _, cam = synth.render_pair(5, "160x120")
    pc, oc = cams(cam)
    for mode in (O.REF32, O.F64):
        a, _ = O.build_cloud(mode, d1, oc)
        b, _ = O.build_cloud(mode, d1, oc)
        n = len(a)
        cov0 = a.get("gaussian_cov").reshape(n, 9).copy()
        mean0 = a.get("gaussian_mean").reshape(n, 3).copy()
        O.cloud_add(a, b, np.eye(4))
        assert len(a) == 2 * n
        removed = O.merge(mode, a, oc, np.eye(4))
        assert removed == n and len(a) == n
        cov = a.get("gaussian_cov").reshape(n, 9)
        tol = 1e-12 if mode == O.F64 else 1e-4
        assert np.max(np.abs(cov - cov0 / 2)) <= tol * np.max(np.abs(cov0))
        assert np.max(np.abs(a.get("gaussian_mean").reshape(n, 3) - mean0)) <= tol * 10


def _gpu_cloud(ctx, cam, depth):
    proj, conv = converter(cam, ctx)
    conv.keepGaussians = True
    c = api.Cloud(ctx)
    conv.compute(c, depth)
    return proj, conv, c


def _compare(ctx, gpu_cloud, ocloud):
    d = gpu_cloud.download()
    mean, cov = gpu_cloud.gaussians()
    n = len(ocloud)
    assert len(d["points"]) == n
    assert np.array_equal(d["points"][:, :3], ocloud.get("points").reshape(n, 4)[:, :3].astype(np.float32))
    assert np.array_equal(mean, ocloud.get("gaussian_mean").reshape(n, 3).astype(np.float32))
    assert np.array_equal(cov.reshape(n, 9), ocloud.get("gaussian_cov").reshape(n, 9).astype(np.float32))


@pytest.mark.gpu
def test_merge_copy_matches_ref32(ctx):
    d1, _, _, cam = synth.render_pair(5, "320x240")
    proj, conv, a = _gpu_cloud(ctx, cam, d1)
    _, _, b = _gpu_cloud(ctx, cam, d1)
    a.add(b, np.eye(4))
    m = api.Merger(ctx)
    m.setDepthImageConverter(conv)
    m.setImageSize(cam["rows"], cam["cols"])
    m.merge(a, np.eye(4))
    pc, oc = cams(cam)
    oa, _ = O.build_cloud(O.REF32, d1, oc)
    ob, _ = O.build_cloud(O.REF32, d1, oc)
    O.cloud_add(oa, ob, np.eye(4))
    removed = O.merge(O.REF32, oa, oc, np.eye(4))
    assert m.removed == removed > 0
    _compare(ctx, a, oa)


@pytest.mark.gpu
def test_scene_fusion_matches_ref32(ctx):
    frames, poses, cam = synth.render_sequence(77, "320x240", n_frames=3, period=200)
    T01 = synth.rel(poses[0], poses[2]).astype(np.float32).astype(np.float64)  # frame 2 -> frame 0
    proj, conv, scene = _gpu_cloud(ctx, cam, frames[0])
    _, _, cur = _gpu_cloud(ctx, cam, frames[2])
    scene.add(cur, T01)
    m = api.Merger(ctx)
    m.setDepthImageConverter(conv)
    m.setImageSize(cam["rows"], cam["cols"])
    m.merge(scene, T01)
    pc, oc = cams(cam)
    os_, _ = O.build_cloud(O.REF32, frames[0], oc)
    oc_, _ = O.build_cloud(O.REF32, frames[2], oc)
    O.cloud_add(os_, oc_, T01)
    removed = O.merge(O.REF32, os_, oc, T01)
    assert m.removed == removed > 1000
    _compare(ctx, scene, os_)
    # the merged cloud still aligns: frame 2 against the fused scene
    al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
    al.computeStatistics = False
    _, _, cur2 = _gpu_cloud(ctx, cam, frames[2])
    al.setReferenceCloud(scene)
    al.setCurrentCloud(cur2)
    al.setInitialGuess(T01)
    al.align()
    er, et = synth.pose_error(al.T(), synth.rel(poses[0], poses[2]))
    assert er < 5e-3 and et < 1e-2, (er, et)


@pytest.mark.gpu
def test_merge_needs_gaussians(ctx):
    d1, _, _, cam = synth.render_pair(5, "160x120")
    proj, conv = converter(cam, ctx)
    c = api.Cloud(ctx)
    conv.compute(c, d1)
    m = api.Merger(ctx)
    m.setDepthImageConverter(conv)
    m.setImageSize(cam["rows"], cam["cols"])
    with pytest.raises(L.NicpError):
        m.merge(c)
