"""The C++ host classes (include/nicp_b200/nicp.hpp): a program written
against the reference's class names compiles with g++, links
libnicp_b200.so, and aligns a pair to bitwise the same pose as the Python
mirror of the same classes."""
import os
import subprocess

import numpy as np
import pytest

from nicp_b200 import synth

from helpers import converter, gpu_cloud, projector

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_caller(tmp_path):
    exe = str(tmp_path / "simple_aligner")
    libdir = os.path.join(ROOT, "nicp_b200")
    cmd = [os.environ.get("NICP_CXX", "g++"), "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "simple_aligner.cpp"), "-L", libdir, "-lnicp_b200",
           "-Wl,-rpath," + libdir, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_header_compiles(built, tmp_path):
    exe = compile_caller(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_caller_matches_python(ctx, tmp_path):
    exe = compile_caller(tmp_path)
    d1, d2, Tgt, cam = synth.render_pair(17, "320x240")
    frames = tmp_path / "frames.bin"
    np.concatenate([d1.ravel(), d2.ravel()]).astype(np.uint16).tofile(frames)
    out = subprocess.run([exe, str(frames), str(cam["rows"]), str(cam["cols"]), repr(cam["fx"]), repr(cam["fy"]),
                          repr(cam["cx"]), repr(cam["cy"])], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    T_cpp = np.array([float(x) for x in lines[0].split()]).reshape(4, 4)
    err, inl, valid, npts = lines[1].split()
    from nicp_b200 import api
    proj, conv = converter(cam, ctx)
    ref, _ = gpu_cloud(ctx, conv, d1, keep_index=False)
    cur, _ = gpu_cloud(ctx, conv, d2, keep_index=False)
    al = api.AlignerProjective(proj, api.Linearizer(ctx), api.CorrespondenceFinderProjective(ctx), ctx)
    al.setReferenceCloud(ref)
    al.setCurrentCloud(cur)
    al.align()
    assert np.array_equal(T_cpp, al.T())
    assert int(inl) == al.inliers() and int(npts) == len(ref)
    assert bool(int(valid)) == al.solutionValid()
