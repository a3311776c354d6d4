"""The 8-wide copy of the tree, on the host: tests/wide_check.cpp is compiled with the library's host
sources (the 4-wide builder and the widening, ebgeometry_b200/csrc/mesh_host.cpp and mesh_wide.cpp)
and checks, for both build methods and several leaf sizes, that the copy holds the 4-wide tree's
leaves and boxes unchanged and prunes a nearest-box search exactly as the 4-wide tree does.  The GPU
side (queries through the copy give the 4-wide results bit for bit) is tests/test_wide_gpu.py."""
import os
import shutil
import subprocess

from conftest import ROOT

CSRC = os.path.join(ROOT, "ebgeometry_b200", "csrc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def test_widened_tree_keeps_leaves_boxes_and_answers(tmp_path):
    exe = str(tmp_path / "wide_check")
    cmd = [CXX, "-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off", f"-I{CSRC}",
           os.path.join(ROOT, "tests", "wide_check.cpp"), os.path.join(CSRC, "mesh_host.cpp"),
           os.path.join(CSRC, "mesh_wide.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(run.stdout)
    assert run.returncode == 0 and "FAIL" not in run.stdout, run.stdout + run.stderr
    assert run.stdout.count("ok ") == 14
