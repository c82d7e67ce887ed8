"""The C++ classes with the reference's solver interface (include/ins_solver_b200/
solvers.hpp): they compile and link against the library here, and on a GPU they
solve pressure, Helmholtz and slip-viscous problems and extrapolate initial guesses."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_check.cpp")
LIBDIR = os.path.join(ROOT, "ins-solver_b200")


def _build(tmp_path):
    exe = str(tmp_path / "shim_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lsipg_b200", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_classes_compile_and_link(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_shim_classes_solve_like_the_reference_drives_them(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
