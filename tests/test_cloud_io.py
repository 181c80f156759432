"""The reference's on-disk formats: .nicp clouds (Cloud::save / Cloud::load,
cloud.cpp:13-150) and trajectory lines (nicp_simple_aligner.cpp:175-181).

The checker here is a Python restatement of the reference writer: it builds
the expected bytes of a binary .nicp file from the cloud's downloaded arrays
(Point, Normal, then the 96-byte Stats: 4x4 column-major, int n,
eigenvalues, bool curvatureComputed at byte 80, float curvature at 84,
zero padding), and the expected text lines with iostream's %g formatting."""
import ctypes as C
import math
import struct

import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth

from helpers import converter


def test_trajectory_line():
    # rotation of 90 degrees about z, translation (1, 2, 3)
    T = np.eye(4, dtype=np.float32)
    T[:3, :3] = [[0, -1, 0], [1, 0, 0], [0, 0, 1]]
    T[:3, 3] = [1, 2, 3]
    line = api.trajectory_line("1305031102.175304", T)
    s = math.sqrt(0.5)
    want = "1305031102.175304 1 2 3 %g %g %g %g\n" % (0.0, 0.0, np.float32(s), np.float32(s))
    assert line == want, (line, want)
    # a rotation of 180 degrees about x takes the largest-diagonal branch
    T2 = np.diag([1, -1, -1, 1]).astype(np.float32)
    assert api.trajectory_line("0", T2) == "0 0 0 0 1 0 0 0\n"


def _record(p, n, rec, kappa, has_stats):
    """Expected bytes of one binary .nicp point (cloud.cpp:125-146)."""
    out = struct.pack("<4f", p[0], p[1], p[2], 1.0) + struct.pack("<4f", n[0], n[1], n[2], 0.0)
    if not has_stats:
        M = np.zeros((4, 4), np.float32)
        nn, ev, comp, curv = 0, (0.0, 0.0, 0.0), 0, 1.0
    else:
        M = np.zeros((4, 4), np.float32)
        M[:3, :3] = rec["U"]
        M[:3, 3] = rec["mean"]
        M[3, 3] = 1.0
        nn, ev = rec["n"], tuple(rec["ev"])
        comp, curv = (1, kappa) if nn > 0 else (0, 1.0)
    stats = M.T.astype("<f4").tobytes() + struct.pack("<i3f", nn, *ev) + bytes([comp, 0, 0, 0]) + \
        struct.pack("<f", curv) + bytes(8)
    assert len(stats) == 96
    return out + stats


@pytest.mark.gpu
@pytest.mark.parametrize("keep_stats", [True, False], ids=["stats", "no_stats"])
def test_binary_nicp_bytes(ctx, tmp_path, keep_stats):
    d1, _, _, cam = synth.render_pair(21, "160x120")
    proj, conv = converter(cam, ctx, keep_stats=keep_stats)
    c = api.Cloud(ctx)
    conv.compute(c, d1)
    T = synth.make_T(synth.rot([0, 1, 0], 0.3), [0.1, -0.2, 0.3]).astype(np.float32)
    f = tmp_path / "c.nicp"
    c.save(f, T, step=1, binary=True)
    raw = f.read_bytes()
    d = c.download(stats=keep_stats)
    n = len(d["points"])
    head, rest = raw.split(b"\n", 1)
    assert head == b"NICPCLOUD %d 1" % n
    line2, body = rest.split(b"\n", 1)
    x = [float(v) for v in line2.split()]
    assert np.allclose(x[:3], [0.1, -0.2, 0.3], atol=1e-6) and abs(x[4] - math.sin(0.15)) < 1e-5
    assert len(body) == 128 * n
    # the stats records as the device keeps them (mean, n) come only with keep_stats
    if keep_stats:
        recs = _stats_records(c, n)
    for i in list(range(0, n, max(1, n // 300))) + [n - 1]:
        rec = recs[i] if keep_stats else None
        want = _record(d["points"][i], d["normals"][i], rec, d["curvature"][i], keep_stats)
        assert body[128 * i:128 * (i + 1)] == want, i


def _stats_records(c, n):
    st = c.stats()
    return [dict(U=st["eigenvectors"][i], mean=st["mean"][i], n=int(st["n"][i]), ev=st["eigenvalues"][i])
            for i in range(n)]


@pytest.mark.gpu
def test_round_trip_and_alignment(ctx, tmp_path):
    d1, d2, Tgt, cam = synth.render_pair(22, "320x240")
    proj, conv = converter(cam, ctx, keep_stats=True)
    ref, cur = api.Cloud(ctx), api.Cloud(ctx)
    conv.compute(ref, d1)
    conv.compute(cur, d2)
    T = synth.make_T(synth.rot([1, 0, 0], -0.2), [0.0, 0.5, -0.1]).astype(np.float32)
    for binary in (True, False):
        f = tmp_path / ("r%d.nicp" % binary)
        ref.save(f, T, 1, binary)
        back = api.Cloud(ctx)
        Tb = back.load(f)
        assert np.allclose(Tb, T, atol=2e-6 if binary else 2e-5)
        a, b = ref.download(stats=True), back.download(stats=True)
        assert len(a["points"]) == len(b["points"])
        tol = 0.0 if binary else 1e-5
        for k in ("points", "normals", "curvature", "eigenvalues", "eigenvectors"):
            x, y = a[k].astype(np.float64), b[k].astype(np.float64)
            if binary and k != "curvature":
                assert np.array_equal(x, y), k
            elif k in ("points", "normals", "eigenvectors"):
                assert np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(x))) + 1e-6, k
        # information matrices are recomputed from the Stats on load
        for k in ("omega_p", "omega_n"):
            x, y = a[k].astype(np.float64), b[k].astype(np.float64)
            scale = np.maximum(np.max(np.abs(x), axis=(1, 2)), 1e-30)
            assert np.max(np.max(np.abs(x - y), axis=(1, 2)) / scale) < (1e-5 if binary else 1e-3), k
        if binary:
            # a loaded cloud aligns like the one it was saved from
            al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
            al.computeStatistics = False
            al.setReferenceCloud(ref)
            al.setCurrentCloud(cur)
            T0 = al.align().copy()
            al.setReferenceCloud(back)
            T1 = al.align()
            er, et = synth.pose_error(T1, T0)
            assert er < 1e-5 and et < 5e-5, (er, et)


@pytest.mark.gpu
def test_step_and_header_count(ctx, tmp_path):
    d1, _, _, cam = synth.render_pair(23, "160x120")
    proj, conv = converter(cam, ctx)
    c = api.Cloud(ctx)
    conv.compute(c, d1)
    n = c.size()
    f = tmp_path / "s.nicp"
    c.save(f, None, 3, True)
    raw = f.read_bytes()
    head, line2, body = raw.split(b"\n", 2)
    # the reference's header counts n / 3 while its loop writes every third point
    assert head == b"NICPCLOUD %d 1" % (n // 3)
    assert len(body) == 128 * ((n + 2) // 3)
    back = api.Cloud(ctx)
    back.load(f)
    assert back.size() == n // 3
    bad = tmp_path / "bad.nicp"
    bad.write_bytes(b"NOTACLOUD 3 1\n0 0 0 0 0 0\n")
    with pytest.raises(L.NicpError):
        api.Cloud(ctx).load(bad)
    # a header that claims more points than the file holds (2^24 here): the
    # records present are loaded, memory follows them (not the header), and
    # the call reports NICP_EINVAL
    short = tmp_path / "short.nicp"
    short.write_bytes(b"NICPCLOUD %d 1\n" % (1 << 24) + line2 + b"\n" + body[:256])
    got = api.Cloud(ctx)
    k = C.c_int(-1)
    rc = ctx.lib.nicp_cloud_load(got.h, str(short).encode(), None, None, C.byref(k))
    assert rc == L.NICP_EINVAL and k.value == 2 and got.size() == 2
