"""Controls of the batched loop (no reference counterpart): the autotuner's
launch shapes and the per-pair early exit.

* Autotuned and default launch shapes give bitwise the same poses (the
  shapes change how work is spread, not what is summed or in which order).
* A pair stops once its pose changes by less than early_exit_eps in an outer
  iteration; its result then differs from the full run by no more than the
  remaining iterations would have moved it, and pairs that converge early
  report fewer iterations."""
import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth

from helpers import converter, gpu_cloud

pytestmark = pytest.mark.gpu

SPECS = [(51, "160x120"), (52, "320x240"), (53, "640x480"), (54, "320x240"), (55, "640x480"), (56, "160x120")]


@pytest.fixture(scope="module")
def batch(ctx):
    refs, curs, cams, truth = [], [], [], []
    for seed, name in SPECS:
        d1, d2, Tgt, cam = synth.render_pair(seed, name, deg=0.5, deg_hi=5.0, meters=0.01, m_hi=0.08)
        proj, conv = converter(cam, ctx)
        refs.append(gpu_cloud(ctx, conv, d1, keep_index=False)[0])
        curs.append(gpu_cloud(ctx, conv, d2, keep_index=False)[0])
        cams.append(proj.camera())
        truth.append(Tgt)
    return refs, curs, cams, truth


def _params(ctx, outer=20, inner=2, eps=0.0):
    prm = L.AlignParams()
    ctx.lib.nicp_default_align_params(prm)
    prm.compute_statistics = 0
    prm.outer_iterations, prm.inner_iterations, prm.early_exit_eps = outer, inner, eps
    return prm


def _run(ctx, batch, prm):
    refs, curs, cams, _ = batch
    corr = api.CorrespondenceFinderProjective(ctx).params()
    lin = api.Linearizer(ctx).params()
    return api.align_batch(ctx, refs, curs, cams, None, corr, lin, prm)


def test_autotuned_shapes_give_identical_results(ctx, batch):
    prm = _params(ctx)
    ctx.set_autotune(False)
    base = _run(ctx, batch, prm)
    # six pairs: fewer than two waves of z-buffer CTAs, so 4 points per thread
    assert ctx.launch_shape()[:2] == (4, 0)
    ctx.set_autotune(True)
    try:
        tuned = _run(ctx, batch, prm)
        ppt, ctas, mixes = ctx.launch_shape()
        assert ppt in (1, 2, 4, 8) and ctas in (0, 2, 3) and mixes >= 1
        again = _run(ctx, batch, prm)  # cached choice, no new trials
        assert ctx.launch_shape() == (ppt, ctas, mixes)
    finally:
        ctx.set_autotune(False)
    for a, b, c in zip(base, tuned, again):
        assert np.array_equal(np.array(a.T), np.array(b.T))
        assert np.array_equal(np.array(a.T), np.array(c.T))
        assert a.inliers == b.inliers == c.inliers


def test_early_exit(ctx, batch):
    full = _run(ctx, batch, _params(ctx))
    early = _run(ctx, batch, _params(ctx, eps=1e-4))
    iters = [r.outer_iterations_run for r in early]
    assert all(r.outer_iterations_run == 20 for r in full)
    assert min(iters) < 20, iters
    for f, e in zip(full, early):
        er, et = synth.pose_error(np.array(e.T).reshape(4, 4), np.array(f.T).reshape(4, 4))
        if e.outer_iterations_run < 20:
            assert er < 2e-3 and et < 2e-3, (er, et, e.outer_iterations_run)
        else:
            assert np.array_equal(np.array(e.T), np.array(f.T))


def test_wide_batch_default_shape_matches_single_pairs(ctx):
    """Eight 640x480 pairs give a z-buffer grid of two waves or more, where
    the default is 8 points per thread; a pair alone runs with 4.  Both must
    give bitwise the same poses (the z-buffer's atomicMin is order-free)."""
    refs, curs, cams = [], [], []
    for seed in range(61, 69):
        d1, d2, _, cam = synth.render_pair(seed, "640x480", deg=0.5, deg_hi=5.0, meters=0.01, m_hi=0.08)
        proj, conv = converter(cam, ctx)
        refs.append(gpu_cloud(ctx, conv, d1, keep_index=False)[0])
        curs.append(gpu_cloud(ctx, conv, d2, keep_index=False)[0])
        cams.append(proj.camera())
    prm = _params(ctx, outer=10, inner=1)
    corr = api.CorrespondenceFinderProjective(ctx).params()
    lin = api.Linearizer(ctx).params()
    ctx.set_autotune(False)
    wide = api.align_batch(ctx, refs, curs, cams, None, corr, lin, prm)
    assert ctx.launch_shape()[:2] == (8, 0)
    for i in range(len(refs)):
        one = api.align_batch(ctx, refs[i:i + 1], curs[i:i + 1], cams[i:i + 1], None, corr, lin, prm)
        assert ctx.launch_shape()[:2] == (4, 0)
        assert np.array_equal(np.array(one[0].T), np.array(wide[i].T))
        assert one[0].inliers == wide[i].inliers


def test_autotuned_stats_shape_gives_identical_clouds(ctx):
    """The build's autotuner (stats kernel: threads per CTA x CTAs per SM)
    leaves every cloud bitwise as the default shape builds it, the count of
    points with a normal included (the trials run the kernel several times)."""
    frames, cam_list = [], []
    for seed, name in [(61, "640x480"), (62, "320x240"), (63, "640x480")]:
        d1, _, _, cam = synth.render_pair(seed, name)
        proj, conv = converter(cam, ctx, keep_stats=True)
        frames.append(d1)
        cam_list.append(proj.camera(cam["rows"], cam["cols"]))
        prm = conv.params()

    def build():
        outs = [api.Cloud(ctx) for _ in frames]
        api.build_batch(ctx, frames, cam_list, prm, outs)
        return [(o.download(stats=True), ctx.lib) for o in outs], outs

    ctx.set_autotune(False)
    base, keep0 = build()
    assert ctx.stats_shape() == (256, 3)
    ctx.set_autotune(True)
    try:
        tuned, keep1 = build()
        shape = ctx.stats_shape()
        assert shape in ((256, 3), (128, 6), (64, 12), (256, 2))
        again, keep2 = build()  # cached choice
        assert ctx.stats_shape() == shape
    finally:
        ctx.set_autotune(False)
    for (a, _), (b, _), (c, _) in zip(base, tuned, again):
        for k in ("points", "normals", "curvature", "omega_p", "omega_n", "eigenvalues", "eigenvectors"):
            assert np.array_equal(a[k], b[k]) and np.array_equal(a[k], c[k]), k
    counts = [[o.normal_count() for o in outs] for outs in (keep0, keep1, keep2)]
    assert counts[0] == counts[1] == counts[2]
    assert counts[0] == [int((np.abs(a["normals"][:, :3]).sum(1) > 0).sum()) for a, _ in base]
