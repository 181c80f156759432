"""The C-ABI boundary, checked without a GPU: the library loads, exports every
function declared in include/*.h, its host-side entry points agree with the
oracle bit for bit, and it refuses to run without an sm_100 device (no CPU
fallback)."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from nicp_b200 import _lib as L
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nicp_[a-z0-9_]+)\s*\(", src)))


def exported(lib_path):
    lib = C.CDLL(lib_path)
    return lib


def test_gpu_library_exports_every_declared_symbol(built):
    lib = exported(L.LIB_PATH)
    names = declared("nicp_gpu.h")
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert sorted(L.SIGNATURES) == names


def test_synth_library_exports(built):
    from nicp_b200 import synth
    lib = exported(synth.SYNTH_PATH)
    for n in declared("nicp_synth.h"):
        assert hasattr(lib, n), n


def test_no_context_without_gpu(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nicp_b200 import Context
    with pytest.raises(L.NicpError):
        Context(0)


def test_defaults_match_reference_constructors(built):
    lib = L.load()
    c = L.Camera()
    lib.nicp_default_camera(C.byref(c))
    assert (c.fx, c.fy, c.cx, c.cy) == (1.0, 1.0, 0.5, 0.5)            # pinholepointprojector.cpp:6-9
    assert (np.float32(c.min_distance), np.float32(c.max_distance)) == (np.float32(0.01), np.float32(6.0))
    assert (np.float32(c.baseline), np.float32(c.alpha)) == (np.float32(0.075), np.float32(0.1))
    p = L.CloudParams()
    lib.nicp_default_cloud_params(C.byref(p))
    assert (p.min_image_radius, p.max_image_radius, p.min_points) == (10, 30, 50)
    assert np.float32(p.curvature_threshold) == np.float32(0.02)
    assert list(p.pim_flat) == [1000.0, np.float32(0.001), np.float32(0.001)]
    assert list(p.nim_nonflat) == [np.float32(0.1), 1.0, 1.0]
    cp = L.CorrParams()
    lib.nicp_default_corr_params(C.byref(cp))
    assert np.float32(cp.inlier_normal_angular_threshold) == np.float32(math.cos(np.float32(math.pi / 6)))
    assert np.float32(cp.flat_curvature_threshold) == np.float32(0.2)
    assert np.float32(cp.inlier_curvature_ratio_threshold) == np.float32(1.3)
    lp = L.LinParams()
    lib.nicp_default_lin_params(C.byref(lp))
    assert (lp.inlier_max_chi2, lp.robust_kernel, lp.z_scaling, lp.scale) == (9000.0, 1, 0, 1.0)
    ap = L.AlignParams()
    lib.nicp_default_align_params(C.byref(ap))
    assert (ap.outer_iterations, ap.inner_iterations, ap.lambda_, ap.min_inliers) == (10, 1, 1000.0, 100)
    assert ap.early_exit_eps == 0.0


@pytest.mark.parametrize("seed", range(6))
def test_projector_matrices_match_oracle(built, seed):
    """KRt / iKRt of _updateMatrices are bit-identical to the REF32 restatement,
    so both sides feed identical matrices to their projections."""
    from nicp_b200 import synth
    rng = np.random.default_rng(seed)
    cam = synth.camera_dict(["160x120", "320x240", "640x480", "1280x720"][seed % 4])
    T = synth.random_offset(rng, 0.5, 20.0, 0.01, 2.0).astype(np.float32)
    scaling = [1.0, 0.5, 2.0][seed % 3]
    c = L.Camera(cam["fx"], cam["fy"], cam["cx"], cam["cy"], scaling, cam["rows"], cam["cols"], 0.01, 6.0, 0.075, 0.1)
    K, iK = np.zeros(16, np.float32), np.zeros(16, np.float32)
    assert L.load().nicp_projector_matrices(C.byref(c), L.fptr(T), L.fptr(K), L.fptr(iK)) == 0
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"], scaling=scaling)
    oK, oiK = O.projector_matrices(O.REF32, oc, T.astype(np.float64))
    assert np.array_equal(K.reshape(4, 4), oK.astype(np.float32))
    assert np.array_equal(iK.reshape(4, 4), oiK.astype(np.float32))


def test_bad_arguments_rejected(built):
    lib = L.load()
    assert lib.nicp_ctx_create(0, None, None) == L.NICP_EINVAL
    assert lib.nicp_projector_matrices(None, None, None, None) == L.NICP_EINVAL


GUARD_PROBE = r"""
#include <cstdio>
#include <stdexcept>
#include <vector>
#include "abi_guard.hpp"

static int entry(int what) {
  NICP_ABI_TRY
  if (what == 1) throw std::bad_alloc();
  if (what == 2) { std::vector<double> v; v.reserve(v.max_size() + 1); }
  if (what == 3) throw std::runtime_error("other");
  return NICP_OK;
  NICP_ABI_CATCH
}

int main() {
  for (int w = 0; w < 4; w++) std::printf("%d ", entry(w));
  return 0;
}
"""


def test_abi_guard_turns_exceptions_into_status(tmp_path):
    """Every C entry point runs inside NICP_ABI_TRY / NICP_ABI_CATCH: an
    allocation failure or an oversized container request comes back as
    NICP_ENOMEM, any other exception as NICP_ESTATE, and nothing escapes."""
    import subprocess
    src = tmp_path / "guard.cpp"
    src.write_text(GUARD_PROBE)
    exe = tmp_path / "guard"
    subprocess.run([os.environ.get("NICP_CXX", "g++"), "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "nicp_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert [int(x) for x in out] == [L.NICP_OK, L.NICP_ENOMEM, L.NICP_ENOMEM, L.NICP_ESTATE]


def test_every_entry_point_is_guarded():
    """Each `extern "C" int` definition in the library's sources opens with
    NICP_ABI_TRY and closes with NICP_ABI_CATCH."""
    csrc = os.path.join(ROOT, "nicp_b200", "csrc")
    for name in ("capi.cu", "cloud_io.cpp", "server.cpp"):
        src = open(os.path.join(csrc, name)).read()
        defs = re.findall(r'^extern "C" int (nicp_\w+)\([^;{]*\)\s*\{\n  NICP_ABI_TRY\n', src, flags=re.M)
        total = re.findall(r'^extern "C" int (nicp_\w+)\([^;{]*\)\s*\{', src, flags=re.M)
        assert total and sorted(defs) == sorted(total), (name, sorted(set(total) - set(defs)))
        assert src.count("NICP_ABI_CATCH") == len(total), name
