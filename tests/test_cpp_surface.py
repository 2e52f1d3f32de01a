"""The C++ drop-in surface (include/*.h: the reference's classes over
libbbk_b200): it compiles and links on any machine; on a GPU its test program
(tests/cpp/test_cpp_surface.cc) must pass, including the block geometry,
permutation, pivot types and factor bits of the reference after boundary
shifts (tests/golden/ref_geometry.txt)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_surface.cc")
FIXTURE = os.path.join(ROOT, "tests", "golden", "ref_geometry.txt")


def _compile(bbk, out: str) -> subprocess.CompletedProcess:
    libdir = os.path.dirname(bbk.LIB_PATH)
    gxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [gxx, "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-L", libdir,
           "-lbbk_b200", f"-Wl,-rpath,{libdir}", "-o", out]
    return subprocess.run(cmd, capture_output=True, text=True)


def test_cpp_surface_compiles_and_links(bbk, tmp_path):
    r = _compile(bbk, str(tmp_path / "t"))
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_surface_runs(cuda, bbk, tmp_path):
    exe = str(tmp_path / "t")
    r = _compile(bbk, exe)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe, FIXTURE], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "passed" in run.stdout
