"""nicp_linearize_noalloc: the linearizer for callers that cannot allocate
device memory (a real-time loop that cannot pay for cudaMalloc's
synchronisation, or a framework that owns all device memory).  Its partial
sums live in a fixed array inside the library, so it must give the same
H, b, error and inliers as nicp_linearize -- and, directly, as the FP64
oracle's linearizer on the same clouds and correspondences -- and two calls
in a row must not see each other's leftovers in that shared array.

This file is collected last on purpose: it must pass both alone in a fresh
process and after every other test."""
import ctypes as C

import numpy as np
import pytest

from nicp_b200 import _lib as L
from nicp_b200 import api, synth

from oracle import oracle as O

from helpers import converter, float_T, gpu_cloud, oracle_cloud_from_gpu, perturb

pytestmark = pytest.mark.gpu


def _noalloc(ctx, ref, cur, pairs, T, lp, threads):
    import torch
    dev_pairs = torch.from_numpy(np.ascontiguousarray(pairs, np.int32).reshape(-1)).cuda()
    out = torch.full((44,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = ctx.lib.nicp_linearize_noalloc(ctx.h, ref.h, cur.h, C.c_void_p(dev_pairs.data_ptr()), len(pairs),
                                        L.fptr(L.f16(T)), C.byref(lp), threads, C.c_void_p(out.data_ptr()))
    assert rc == L.NICP_OK, rc
    ctx.synchronize()
    o = out.cpu().numpy()
    return o[:36].reshape(6, 6), o[36:42], o[42], int(o[43])


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_noalloc_linearize_matches_nicp_linearize(ctx):
    d1, d2, Tgt, cam = synth.render_pair(23, "320x240")
    proj, conv = converter(cam, ctx)
    ref, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
    cur, _ = gpu_cloud(ctx, conv, d2, keep_index=False)
    proj.setTransform(np.eye(4))
    ci, _ = proj.project(cur)
    proj.setTransform(Tgt)
    ri, _ = proj.project(ref)
    cf = api.CorrespondenceFinderProjective(ctx)
    cf.setReferenceIndexImage(ri)
    cf.setCurrentIndexImage(ci)
    Tinv = np.linalg.inv(float_T(Tgt)).astype(np.float32)
    pairs = cf.compute(ref, cur, Tinv)
    assert len(pairs) > 1000
    lin = api.Linearizer(ctx)
    lp = lin.params()
    oref = oracle_cloud_from_gpu(O.F64, ref.download())
    ocur = oracle_cloud_from_gpu(O.F64, cur.download())
    # two calls in a row with different inputs: the second must not inherit
    # anything from the first through the shared partial-sum array
    T2 = (np.linalg.inv(float_T(Tgt)) @ perturb(4, 0.5, 0.01)).astype(np.float32)
    for sub, T, threads in [(pairs, Tinv, 1), (pairs[: len(pairs) // 2 + 7], T2, 3)]:
        lin.setT(T)
        lin.update(ref, cur, sub, parity_threads=threads)
        H, b, err, inl = _noalloc(ctx, ref, cur, sub, T, lp, threads)
        assert inl == lin.inliers()
        assert _rel(H, lin.H()) < 1e-5 and _rel(b, lin.b()) < 1e-5
        assert abs(err - lin.error()) <= 1e-5 * abs(lin.error())
        # against the FP64 oracle (with threads > 1 the last K % threads
        # correspondences are dropped, as the reference drops them): H and the
        # error within 1e-5 relative; b within 1e-5 relative away from the
        # solution (T2), while at the true pose (Tinv) b is the small remainder
        # of terms that cancel, so there the bar is on what b is for: the
        # Gauss-Newton step H^-1 b moves by less than 1e-7 (rad, m), a hundredth
        # of the pose bar
        kk = (len(sub) // threads) * threads
        Ho, bo, erro, inlo = O.linearize(O.F64, oref, ocur, sub[:kk], T.astype(np.float64))
        assert inl == inlo
        assert _rel(H, Ho) < 1e-5, _rel(H, Ho)
        assert abs(err - erro) <= 1e-5 * abs(erro)
        step_diff = np.abs(np.linalg.solve(Ho, b - bo)).max()
        assert step_diff < 1e-7, step_diff
        if T is T2:
            assert _rel(b, bo) < 1e-5, _rel(b, bo)


def test_noalloc_rejects_oversized_list(ctx):
    d1, _, _, cam = synth.render_pair(24, "160x120")
    proj, conv = converter(cam, ctx)
    c, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
    import torch
    lp = api.Linearizer(ctx).params()
    T = np.eye(4, dtype=np.float32)
    # real buffers of the oversized length (no fake addresses): should the
    # host's size check ever regress, the kernels read valid (empty) pairs
    # and their own tile bound keeps them inside the partial-sum array, so
    # the regression shows up as this assertion, not as a GPU fault
    n = L.NICP_LINEARIZE_NOALLOC_MAX_PAIRS + 1
    dev_pairs = torch.full((2 * n,), -1, dtype=torch.int32, device="cuda")
    out = torch.zeros((44,), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = ctx.lib.nicp_linearize_noalloc(ctx.h, c.h, c.h, C.c_void_p(dev_pairs.data_ptr()), n, L.fptr(T), C.byref(lp),
                                        1, C.c_void_p(out.data_ptr()))
    ctx.synchronize()
    assert rc == L.NICP_EINVAL
