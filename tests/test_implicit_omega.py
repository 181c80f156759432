"""Clouds built with the converter's structured information matrices and
without Stats keep Omega implicit: the stats kernel does not write the
matrices (d1 I + (d0 - d1) n n^T from the normal, the class code and the
cloud's (d0, d1) per class), and the library writes them out only for a
reader that needs them (downloads, the list-mode linearizer, Cloud::add with
a cloud whose matrices are explicit).  These tests hold the implicit form to
the explicit one the Stats-keeping build writes, through downloads,
transforms, additions and the list-mode linearizer."""
import numpy as np
import pytest

from nicp_b200 import api, synth

from helpers import converter, float_T

pytestmark = pytest.mark.gpu


def _rel_rows(a, b):
    a = a.reshape(len(a), -1).astype(np.float64)
    b = b.reshape(len(b), -1).astype(np.float64)
    scale = np.maximum(np.max(np.abs(b), axis=1), 1e-30)
    return float(np.max(np.max(np.abs(a - b), axis=1) / scale))


def _twins(ctx, seed=31, name="320x240"):
    d1, d2, Tgt, cam = synth.render_pair(seed, name)
    _, lazy_conv = converter(cam, ctx)
    _, full_conv = converter(cam, ctx, keep_stats=True)
    a, b = api.Cloud(ctx), api.Cloud(ctx)
    lazy_conv.compute(a, d1)
    full_conv.compute(b, d1)
    return a, b, d1, d2, Tgt, cam


def _check_same_omega(da, db, tol):
    assert np.array_equal(da["points"], db["points"])
    assert np.array_equal(da["normals"], db["normals"])
    for k in ("omega_p", "omega_n"):
        assert _rel_rows(da[k], db[k]) < tol, (k, _rel_rows(da[k], db[k]))
        # the class (flat / non-flat) is the same everywhere
        assert np.array_equal(np.trace(da[k].reshape(-1, 3, 3), axis1=1, axis2=2) > 100.0,
                              np.trace(db[k].reshape(-1, 3, 3), axis1=1, axis2=2) > 100.0)


def test_implicit_omega_matches_the_explicit_build(ctx):
    a, b, *_ = _twins(ctx)
    da, db = a.download(), b.download()
    # the explicit build rounds Omega from the double eigenvector, the
    # implicit one from the float normal: a few float ulps apart
    _check_same_omega(da, db, 1e-6)
    # downloading twice gives the same matrices
    da2 = a.download()
    for k in ("omega_p", "omega_n"):
        assert np.array_equal(da[k], da2[k])


def test_implicit_omega_follows_a_transform(ctx):
    a, b, *_ = _twins(ctx, seed=32)
    T = synth.make_T(synth.rot([0.3, 1.0, -0.2], 0.4), [0.1, -0.2, 0.3]).astype(np.float32)
    a.transformInPlace(T)
    b.transformInPlace(T)
    # the implicit form is rebuilt from the rotated normal, the explicit one
    # rotated as R Omega R^T in float
    _check_same_omega(a.download(), b.download(), 1e-5)


def test_add_with_explicit_and_implicit_parts(ctx):
    a, b, *_ = _twins(ctx, seed=33)
    da, db = a.download(), b.download()
    for first, second, d_first, d_second in ((a, b, da, db), (b, a, db, da)):
        scene = api.Cloud(ctx)
        scene.add(first)
        scene.add(second)
        ds = scene.download()
        n = len(d_first["points"])
        for k in ("omega_p", "omega_n"):
            assert np.array_equal(ds[k][:n], d_first[k]), k
            assert np.array_equal(ds[k][n:], d_second[k]), k
    # two implicit parts stay implicit and download as each part does
    a2, _, *_ = _twins(ctx, seed=34)
    scene = api.Cloud(ctx)
    scene.add(a)
    scene.add(a2)
    ds, da2 = scene.download(), a2.download()
    for k in ("omega_p", "omega_n"):
        assert np.array_equal(ds[k], np.concatenate([da[k], da2[k]])), k


def test_list_linearizer_on_implicit_and_explicit_clouds(ctx):
    """The linearizer over a correspondence list reads the current cloud's
    matrices: on the implicit twin it must give the explicit twin's H and b."""
    d1, d2, Tgt, cam = synth.render_pair(35, "320x240")
    proj, lazy_conv = converter(cam, ctx)
    _, full_conv = converter(cam, ctx, keep_stats=True)
    ref = api.Cloud(ctx)
    lazy_conv.compute(ref, d1)
    a, b = api.Cloud(ctx), api.Cloud(ctx)
    lazy_conv.compute(a, d2)
    full_conv.compute(b, d2)
    proj.setTransform(np.eye(4))
    ci, _ = proj.project(a)
    proj.setTransform(Tgt)
    ri, _ = proj.project(ref)
    cf = api.CorrespondenceFinderProjective(ctx)
    cf.setReferenceIndexImage(ri)
    cf.setCurrentIndexImage(ci)
    Tinv = np.linalg.inv(float_T(Tgt)).astype(np.float32)
    out = []
    for cur in (a, b):  # a first: its matrices are still implicit here
        pairs = cf.compute(ref, cur, Tinv)
        lin = api.Linearizer(ctx)
        lin.setT(Tinv)
        lin.update(ref, cur, pairs)
        out.append((lin.H().copy(), lin.b().copy(), lin.inliers(), len(pairs)))
    (Ha, ba, ia, na), (Hb, bb, ib, nb) = out
    assert na == nb and na > 1000 and ia == ib
    assert np.linalg.norm(Ha - Hb) <= 1e-5 * np.linalg.norm(Hb)
    # at the true pose b is the small remainder of cancelling terms: bound
    # the Gauss-Newton step it gives instead
    assert np.abs(np.linalg.solve(Hb, ba - bb)).max() < 1e-7


def test_merge_keeps_implicit_omega_consistent(ctx):
    """The merger moves points inside a cloud (its information matrices move
    with them, or stay implicit): implicit and explicit twins merged the same
    way give the same points and normals, and Omega a few ulps apart."""
    d1, _, _, cam = synth.render_pair(36, "320x240")
    out = []
    for keep in (False, True):
        proj, conv = converter(cam, ctx, keep_stats=keep)
        conv.keepGaussians = True
        a, b = api.Cloud(ctx), api.Cloud(ctx)
        conv.compute(a, d1)
        conv.compute(b, d1)
        a.add(b, np.eye(4))
        m = api.Merger(ctx)
        m.setDepthImageConverter(conv)
        m.setImageSize(cam["rows"], cam["cols"])
        m.merge(a, np.eye(4))
        assert m.removed > 0
        out.append((a.download(), m.removed))
    (da, ra), (db, rb) = out
    assert ra == rb
    _check_same_omega(da, db, 1e-6)
