"""The drop-in C++ interface (focalors_poisson_b200/cpp/) on the CPU: it compiles, its tree bookkeeping
(root choice and solve levels, reference base/domain/geometry_tree.hpp) matches the reference's on every
golden composite case, geometry misuse raises the reference's errors, and a solve without a GPU fails
loudly instead of falling back to the CPU."""
import os

import pytest

import dropin_cases as DC
from golden_io import COMPOSITE_CASES, load
from focalors_poisson_b200 import build
from oracle import refpath


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    return DC.driver(tmp_path_factory.mktemp("dropin"))


@pytest.mark.parametrize("name", COMPOSITE_CASES)
def test_tree_matches_reference(exe, tmp_path, name):
    case = str(tmp_path / "case.txt")
    geo = DC.write_case(case, name)
    r = DC.run(exe, case, tree_only=True)
    assert r.returncode == 0, r.stdout + r.stderr
    root, levels, _ = DC.parse(r.stdout, geo)
    z = load(name)
    assert root == int(z["root"])
    assert levels == [int(v) for v in z["levels"]]


def test_disconnected_geometry_rejected(exe, tmp_path):
    case = tmp_path / "case.txt"
    case.write_text("2\n4 4 0.1 0.1 0 0 0 0\n4 4 0.1 0.1 0 0 0 0\n0\n")
    r = DC.run(exe, str(case), tree_only=True)
    assert r.returncode == 3 and "Geometry is not single connected" in r.stdout


def test_cycle_rejected(exe, tmp_path):
    case = tmp_path / "case.txt"
    case.write_text("4\n" + "4 4 0.1 0.1 0 0 0 0\n" * 4 + "4\n0 1 1\n0 3 2\n1 3 3\n2 1 3\n")
    r = DC.run(exe, str(case), tree_only=True)
    assert r.returncode == 3 and "cycle" in r.stdout.lower()


def test_solve_without_device_fails_loudly(exe, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    case = str(tmp_path / "case.txt")
    DC.write_case(case, "lt_shape_2.npz")
    r = DC.run(exe, case)
    assert r.returncode == 3 and "no CUDA device" in r.stdout


def test_library_exports_interface():
    lib = build.build_dropin()
    syms = os.popen(f"nm -D --defined-only {lib}").read()
    for s in ("ConcatPoissonSolver2D5solve", "ConcatPoissonSolver2D13set_parameter", "PoissonSolver2D5solve",
              "Geometry2D7connect", "Variable2D16set_center_field"):
        assert s in syms, s


REFERENCE = refpath.reference_dir()


@pytest.mark.skipif(not refpath.available() or not os.path.exists(
    os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libfpref.so")),
    reason="needs the reference sources and the oracle library built from them")
@pytest.mark.parametrize("case", ["variable_case.cpp", "variable3d_case.cpp"])
def test_host_data_model_matches_reference(tmp_path, case):
    """Geometry2D / Variable2D (variable_case.cpp) and Geometry3D / Variable3D (variable3d_case.cpp) host
    bookkeeping (sizes propagated by connect, axis offsets, tree root and levels, boundary-type overrides and
    their errors, set_value at cell centres, set_buffer at ghost cells, boundary values, corners) prints
    identically through the reference's own sources and through the drop-in layer."""
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "tests", "cases", case)
    ours = build.compile_driver(src, str(tmp_path / "ours"))
    refexe = str(tmp_path / "ref")
    lib = os.path.join(root, "oracle", "_ref")
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-I" + os.path.join(root, "oracle", "shim"), "-I" + REFERENCE,
           "-include", os.path.join(REFERENCE, "base", "pch.h"), src, "-o", refexe, "-L" + lib, "-lfpref",
           "-Wl,-rpath," + lib]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    a = subprocess.run([ours], capture_output=True, text=True, timeout=60)
    b = subprocess.run([refexe], capture_output=True, text=True, timeout=60)
    assert a.returncode == 0 and b.returncode == 0, (a.stdout[-500:], b.stdout[-500:])
    assert a.stdout == b.stdout

