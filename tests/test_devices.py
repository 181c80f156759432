"""Contexts and devices: every call on a context runs on the context's GPU
and gives the calling thread its previous current device back.

On a one-GPU box only the restore half can be observed (the thread's device
stays 0); the two-GPU tests run where a second GPU exists and are skipped
otherwise."""
import ctypes as C
import threading

import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth

from helpers import converter, gpu_cloud

pytestmark = pytest.mark.gpu


def _align_on(device, d1, d2, cam, out, key):
    import torch
    ctx = api.Context(device)
    try:
        proj, conv = converter(cam, ctx)
        ref, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
        cur, _ = gpu_cloud(ctx, conv, d2, keep_index=False)
        al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
        al.computeStatistics = False
        al.setReferenceCloud(ref)
        al.setCurrentCloud(cur)
        al.align()
        out[key] = (al.T(), al.inliers(), torch.cuda.current_device())
    finally:
        ctx.close()


def test_device_guard_keeps_callers_device():
    """Creating a context, building, aligning and destroying it leave the
    calling thread's current device where it was."""
    import torch
    torch.cuda.set_device(0)
    d1, d2, _, cam = synth.render_pair(71, "160x120")
    out = {}
    _align_on(0, d1, d2, cam, out, "a")
    assert torch.cuda.current_device() == 0
    assert out["a"][2] == 0


@pytest.mark.skipif("__import__('torch').cuda.device_count() < 2", reason="needs two GPUs")
def test_contexts_on_two_gpus():
    """The same pair aligned by contexts on GPUs 0 and 1, from two threads
    whose current device is 0: identical poses, and each thread's current
    device is still 0 afterwards."""
    import torch
    d1, d2, _, cam = synth.render_pair(72, "320x240")
    out = {}
    th = [threading.Thread(target=_align_on, args=(dev, d1, d2, cam, out, dev)) for dev in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert set(out) == {0, 1}
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    assert out[0][2] == 0 and out[1][2] == 0


@pytest.mark.skipif("__import__('torch').cuda.device_count() < 2", reason="needs two GPUs")
def test_noalloc_refuses_another_current_device():
    """The allocation-free linearizer switches no device: with GPU 0 current
    it refuses a context of GPU 1 (NICP_ESTATE) before touching memory."""
    import torch
    torch.cuda.set_device(0)
    ctx = api.Context(1)
    try:
        d1, _, _, cam = synth.render_pair(73, "160x120")
        proj, conv = converter(cam, ctx)
        c, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
        with torch.cuda.device(1):
            pairs = torch.zeros((2,), dtype=torch.int32, device="cuda:1")
            out = torch.zeros((44,), dtype=torch.float64, device="cuda:1")
        lp = api.Linearizer(ctx).params()
        T = np.eye(4, dtype=np.float32)
        rc = ctx.lib.nicp_linearize_noalloc(ctx.h, c.h, c.h, C.c_void_p(pairs.data_ptr()), 1, L.fptr(T), C.byref(lp),
                                            1, C.c_void_p(out.data_ptr()))
        assert rc == L.NICP_ESTATE
        assert torch.cuda.current_device() == 0
    finally:
        ctx.close()
