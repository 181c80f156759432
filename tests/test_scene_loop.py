"""The frame-to-scene odometry loop of nicp_aligner.cpp:135-209 on the CUDA
path, step by step against the oracle:

  project the scene into the last view (scaled depth + index image), rebuild
  a subscene cloud from that depth (DepthImageConverter::compute), align the
  new frame's cloud against it from the identity, accumulate the pose, add
  the frame to the scene (Cloud::add) and merge it in that view
  (Merger::merge).

The oracle (REF32, the reference's float arithmetic) runs the same loop fed
with the CUDA path's pose at every step, so that both scenes evolve from the
same inputs: the projected depth and index images, the subscene points and
the merged scene must then be bit-exact, and every pose within 1e-5 rad /
0.05 mm of the FP64 oracle loop run on the same two clouds."""
import numpy as np
import pytest

from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import cams, converter, oracle_cloud_from_gpu

pytestmark = pytest.mark.gpu


def test_frame_to_scene_loop(ctx):
    frames, poses, cam = synth.render_sequence(91, "320x240", n_frames=5, period=200)
    proj, conv = converter(cam, ctx)
    conv.keepGaussians = True
    pc, oc = cams(cam)
    merger = api.Merger(ctx)
    merger.setDepthImageConverter(conv)
    merger.setImageSize(cam["rows"], cam["cols"])
    scene = api.Cloud(ctx)
    conv.compute(scene, frames[0])
    oscene, _ = O.build_cloud(O.REF32, frames[0], oc)
    sceneT = np.eye(4, dtype=np.float32)
    merger.merge(scene, sceneT)
    O.merge(O.REF32, oscene, oc, sceneT.astype(np.float64))
    worst = 0.0
    for k in range(1, len(frames)):
        cloud = api.Cloud(ctx)
        conv.compute(cloud, frames[k])
        ocloud, _ = O.build_cloud(O.REF32, frames[k], oc)
        # the scene seen from the last view
        proj.setTransform(sceneT)
        gidx, gdepth = proj.project(scene)
        oidx, odepth = O.project(O.REF32, oscene, oc, sceneT.astype(np.float64))
        assert np.array_equal(gidx, oidx), k
        assert np.array_equal(gdepth, odepth.astype(np.float32)), k
        sub = api.Cloud(ctx)
        conv.compute(sub, gdepth)
        osub, _ = O.build_cloud_f32(O.REF32, gdepth, oc)
        gs = sub.download()
        assert len(gs["points"]) == len(osub) > 1000, k
        assert np.array_equal(gs["points"], osub.get("points").astype(np.float32)), k
        # align the frame against the subscene from the identity
        al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
        al.computeStatistics = False
        al.setReferenceCloud(sub)
        al.setCurrentCloud(cloud)
        al.align()
        T = al.T()
        r = O.align(O.F64, oracle_cloud_from_gpu(O.F64, gs), oracle_cloud_from_gpu(O.F64, cloud.download()), oc)
        er, et = synth.pose_error(T, r["T"])
        worst = max(worst, er)
        assert er < 1e-5 and et < 5e-5, (k, er, et)
        # accumulate, add and merge (both loops with the CUDA path's pose)
        sceneT = (sceneT.astype(np.float64) @ T).astype(np.float32)
        sceneT[3] = [0, 0, 0, 1]
        scene.add(cloud, sceneT)
        merger.merge(scene, sceneT)
        O.cloud_add(oscene, ocloud, sceneT.astype(np.float64))
        removed = O.merge(O.REF32, oscene, oc, sceneT.astype(np.float64))
        assert merger.removed == removed, k
        d = scene.download()
        assert np.array_equal(d["points"][:, :3], oscene.get("points")[:, :3].astype(np.float32)), k
    # the loop tracks the trajectory
    er, et = synth.pose_error(sceneT.astype(np.float64), synth.rel(poses[0], poses[-1]))
    print("frame-to-scene: worst step vs F64 %.3g rad; end pose vs truth %.3g rad %.3g m" % (worst, er, et))
    assert er < 5e-3 and et < 1e-2
