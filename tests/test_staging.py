"""Depth frames reach the build kernels by several routes: device frames
that are packed and 16-byte aligned are read in place; host frames, pitched
frames and unaligned device frames are first copied into a staging region
(on a separate copy stream, chunk by chunk, overlapped with the build of
earlier chunks).  Every route must give bitwise the same cloud and index
image as the in-place one, for u16 and float depth, single frames and
batches that span several staging chunks."""
import ctypes as C

import numpy as np
import pytest
import torch

from nicp_b200 import _lib as L
from nicp_b200 import api, synth

from helpers import converter

pytestmark = pytest.mark.gpu


def _build_one(ctx, conv, cam_c, ptr, rows, cols, pitch, on_device, f32=False):
    cloud = api.Cloud(ctx)
    idx = np.zeros((rows, cols), np.int32)
    fn = ctx.lib.nicp_cloud_from_depth_f32 if f32 else ctx.lib.nicp_cloud_from_depth_u16
    ctx.check(fn(ctx.h, C.c_void_p(ptr), rows, cols, pitch, 1 if on_device else 0, C.byref(cam_c),
                 C.byref(conv.params()), None, cloud.h, L.iptr(idx)))
    return cloud, idx


def _same(a, b):
    da, db = a.download(), b.download()
    assert len(da["points"]) == len(db["points"])
    for k in ("points", "normals", "curvature", "omega_p", "omega_n"):
        assert np.array_equal(da[k], db[k]), k


@pytest.mark.parametrize("dtype", ["u16", "f32"])
def test_single_frame_routes_agree(ctx, dtype):
    d16, _, _, cam = synth.render_pair(71, "320x240")
    proj, conv = converter(cam, ctx)
    rows, cols = d16.shape
    cam_c = proj.camera(rows, cols)
    f32 = dtype == "f32"
    d = (d16.astype(np.float32) * np.float32(0.001)) if f32 else d16
    d = np.ascontiguousarray(d)
    esz = d.itemsize
    # in place: packed, aligned device frame
    dev = torch.from_numpy(d.view(np.int16) if not f32 else d).cuda()
    ref, ref_idx = _build_one(ctx, conv, cam_c, dev.data_ptr(), rows, cols, 0, True, f32)
    assert np.count_nonzero(ref_idx >= 0) > 10000
    # host, packed
    c1, i1 = _build_one(ctx, conv, cam_c, d.ctypes.data, rows, cols, 0, False, f32)
    # host, pitched (three spare elements per row)
    hp = np.zeros((rows, cols + 3), d.dtype)
    hp[:, :cols] = d
    c2, i2 = _build_one(ctx, conv, cam_c, hp.ctypes.data, rows, cols, (cols + 3) * esz, False, f32)
    # device, unaligned start (one element in)
    flat = torch.zeros(rows * cols + 1, dtype=dev.dtype, device="cuda")
    flat[1:] = dev.reshape(-1)
    c3, i3 = _build_one(ctx, conv, cam_c, flat.data_ptr() + esz, rows, cols, 0, True, f32)
    # device, pitched
    dp = torch.zeros((rows, cols + 5), dtype=dev.dtype, device="cuda")
    dp[:, :cols] = dev
    c4, i4 = _build_one(ctx, conv, cam_c, dp.data_ptr(), rows, cols, (cols + 5) * esz, True, f32)
    torch.cuda.synchronize()
    for c, i in ((c1, i1), (c2, i2), (c3, i3), (c4, i4)):
        assert np.array_equal(i, ref_idx)
        _same(c, ref)


def test_host_batch_across_staging_chunks(ctx):
    """A host batch of 70 frames is staged in several 32-frame chunks whose
    copies overlap the build of earlier chunks; it must equal the same batch
    built from device memory, frame by frame."""
    frames, poses, cam = synth.render_sequence(72, "160x120", n_frames=70)
    proj, conv = converter(cam, ctx)
    cam_c = proj.camera(cam["rows"], cam["cols"])
    prm = conv.params()
    n = len(frames)
    host = [np.ascontiguousarray(f) for f in frames]
    on_host = [api.Cloud(ctx) for _ in range(n)]
    api.build_batch(ctx, host, [cam_c] * n, prm, on_host)
    dev = torch.from_numpy(np.stack(host).view(np.int16)).cuda()
    P = cam["rows"] * cam["cols"]
    ptrs = [(dev.data_ptr() + 2 * P * i, cam["rows"], cam["cols"]) for i in range(n)]
    on_dev = [api.Cloud(ctx) for _ in range(n)]
    api.build_batch(ctx, ptrs, [cam_c] * n, prm, on_dev, on_device=True)
    torch.cuda.synchronize()
    for a, b in zip(on_host, on_dev):
        _same(a, b)
    # and again: the staging region and copy events are reused across calls
    api.build_batch(ctx, host, [cam_c] * n, prm, on_host)
    for a, b in zip(on_host, on_dev):
        _same(a, b)


def test_short_row_pitch_rejected(ctx):
    """A row pitch below the row width is an argument error (NICP_EINVAL),
    caught before any copy; the context stays usable."""
    d16, _, _, cam = synth.render_pair(73, "160x120")
    proj, conv = converter(cam, ctx)
    rows, cols = d16.shape
    cam_c = proj.camera(rows, cols)
    d = np.ascontiguousarray(d16)
    cloud = api.Cloud(ctx)
    rc = ctx.lib.nicp_cloud_from_depth_u16(ctx.h, C.c_void_p(d.ctypes.data), rows, cols, 2 * cols - 2, 0,
                                           C.byref(cam_c), C.byref(conv.params()), None, cloud.h, None)
    assert rc == L.NICP_EINVAL
    _, idx = _build_one(ctx, conv, cam_c, d.ctypes.data, rows, cols, 0, False)
    assert np.count_nonzero(idx >= 0) > 1000
