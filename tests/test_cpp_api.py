"""The C++ drop-in classes (ebgeometry_b200/include/EBGeometry_B200.hpp): a C++ caller compiles
against them standalone and, where the reference sources exist, with the reference's own
SignedDistanceFunction<double> as the base class; on a GPU the example runs and its single-point
value() agrees with the batched call."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

import oracle

EXAMPLE = os.path.join(ROOT, "ebgeometry_b200", "examples", "meshsdf_example.cpp")
LIBDIR = os.path.join(ROOT, "ebgeometry_b200")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
REFERENCE = oracle.reference_dir()


def compile_example(out, extra=(), link=True):
    cmd = [CXX, "-std=c++17", "-O1", f"-I{ROOT}", *extra, EXAMPLE]
    cmd += [f"-L{LIBDIR}", "-lebgb200", f"-Wl,-rpath,{LIBDIR}", "-o", out] if link else ["-c", "-o", out]
    return subprocess.run(cmd, capture_output=True, text=True)


def test_example_compiles_and_links(tmp_path):
    r = compile_example(str(tmp_path / "ex"))
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(REFERENCE is None, reason="reference sources not present on this host (EBG_REFERENCE_DIR)")
def test_classes_derive_from_the_reference_interface(tmp_path):
    r = compile_example(str(tmp_path / "ex.o"), ["-DEBGEOMETRY_B200_WITH_REFERENCE", f"-I{REFERENCE}"], link=False)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_example_runs(tmp_path):
    exe = str(tmp_path / "ex")
    r = compile_example(exe)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0 and "ok" in run.stdout, run.stdout + run.stderr
