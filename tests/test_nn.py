"""Nearest-neighbour association (CorrespondenceFinderNN,
correspondencefindernn.cpp:44-97) and AlignerNN (alignernn.cpp:21-118).

The reference asks FLANN for an approximate nearest neighbour; the CUDA path
and the oracle both compute the exact one (ties: lowest index), so the
correspondence lists are compared bit for bit against the REF32 oracle on
identical clouds and transforms, and the aligner against the FP64 oracle
loop on identical clouds."""
import numpy as np
import pytest

from nicp_b200 import api, synth
from oracle import oracle as O

from helpers import converter, float_T, gpu_cloud, oracle_cloud_from_gpu, perturb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clouds(ctx):
    d1, d2, Tgt, cam = synth.render_pair(31, "320x240", deg=2.0, meters=0.03)
    proj, conv = converter(cam, ctx)
    ref, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
    cur, _ = gpu_cloud(ctx, conv, d2, keep_index=False)
    return ref, cur, Tgt


@pytest.mark.parametrize("scaling,demoted", [(1.0, False), (0.25, False), (1.0, True)])
def test_nn_correspondences_bitexact(ctx, clouds, scaling, demoted):
    ref, cur, Tgt = clouds
    T = np.linalg.inv(float_T(Tgt @ perturb(3, 0.5, 0.01))).astype(np.float32)
    cf = api.CorrespondenceFinderNN(ctx)
    cf.setNormalScaling(scaling)
    cf.setDemotedToGICP(demoted)
    gp = cf.compute(ref, cur, T)
    oref = oracle_cloud_from_gpu(O.REF32, ref.download())
    ocur = oracle_cloud_from_gpu(O.REF32, cur.download())
    prm = O.align_params(corr_demoted_to_gicp=1 if demoted else 0)
    op = O.correspond_nn(O.REF32, oref, ocur, T.astype(np.float64), scaling, prm)
    assert len(gp) > 1000
    assert np.array_equal(gp, op)


def test_align_nn_vs_f64(ctx, clouds):
    ref, cur, Tgt = clouds
    cf = api.CorrespondenceFinderNN(ctx)
    al = api.AlignerNN(None, api.Linearizer(ctx), cf, ctx)
    al.computeStatistics = True
    al.setOuterIterations(10)
    al.setReferenceCloud(ref)
    al.setCurrentCloud(cur)
    T = al.align()
    oref = oracle_cloud_from_gpu(O.F64, ref.download())
    ocur = oracle_cloud_from_gpu(O.F64, cur.download())
    r = O.align_nn(O.F64, oref, ocur, statistics=True)
    er, et = synth.pose_error(T, r["T"])
    assert er < 1e-4 and et < 1e-4, (er, et)
    assert al.solutionValid() == bool(r["solution_valid"])
    et_er = synth.pose_error(T, Tgt)
    assert et_er[0] < 1e-2 and et_er[1] < 3e-2, et_er
