"""GPU parity of the drop-in C++ interface (focalors_poisson_b200/cpp/ over libfpb200): my own driver
(tests/cases/composite_case.cpp) on every golden composite case, and the reference's own validation drivers
(case/validation/2d/{poisson_solver,concat_solver}_reference.cpp, compiled unchanged against the drop-in
headers when the reference sources were present at build time) against the outputs of the reference."""
import os
import subprocess

import numpy as np
import pytest

import dropin_cases as DC
from golden_io import COMPOSITE_CASES, composite_case, load, rel_l2, tight_outputs
from focalors_poisson_b200 import build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    return DC.driver(tmp_path_factory.mktemp("dropin"))


@pytest.mark.parametrize("name", COMPOSITE_CASES)
def test_dropin_composite(exe, tmp_path, name):
    """Same criteria as the C-ABI test of the default (interface GMRES) solve: within the reference's own
    distance from its converged answer at the case's tol, and within 1e-12 of it when driven to 1e-15."""
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    tight = tight_outputs(name)
    own_err = rel_l2(outs, tight)
    case = str(tmp_path / "case.txt")
    DC.write_case(case, name)
    r = DC.run(exe, case)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got_root, _, fields = DC.parse(r.stdout, geo)
    assert got_root == root
    assert rel_l2(fields, outs) <= max(1e-12, 3.0 * own_err), (name, own_err, rel_l2(fields, outs))
    DC.write_case(case, name, tol=1e-15)
    r = DC.run(exe, case)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert rel_l2(DC.parse(r.stdout, geo)[2], tight) <= 1e-12, name


def _reference_driver(name):
    path = os.path.join(build.CASES, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} was not built (the reference sources were absent at build time)")
    return path


def _printed(a, b):
    """field2::print writes 6 significant digits: agreement to that precision."""
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    np.testing.assert_allclose(a, b, rtol=6e-6, atol=1e-9 * max(1.0, float(np.abs(b).max())))


def test_reference_poisson_driver_unchanged():
    exe = _reference_driver("poisson_solver_reference")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    blocks = DC.parse_printed_blocks(r.stdout)
    z = load("poisson.npz")
    assert len(blocks) == len(z["combos"])
    for c, blk in enumerate(blocks):
        _printed(blk, z[f"fixture_{c}"])


def test_reference_concat_driver_unchanged():
    exe = _reference_driver("concat_solver_reference")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    pre, post = r.stdout.split("-----------solve---------------")
    z = load("concat_fixture6.npz")
    before, after = DC.parse_printed_blocks(pre), DC.parse_printed_blocks(post)
    assert len(before) == len(after) == 6
    for d in range(6):
        np.testing.assert_array_equal(before[d], z[f"rhs_{d}"])
        _printed(after[d], z[f"out_{d}"])


def test_dropin_concat3d_case(tmp_path):
    """tests/cases/variable3d_case.cpp (Geometry3D / Variable3D / ConcatPoissonSolver3D of the reference's API,
    four boxes in an L with a box on top) solved through the drop-in layer: per box the solution's sum, norm,
    first and last values equal the reference's own run of the same file (GMRES(20, 1e-13, 100) in both, so the
    two answers differ by the solvers' residual tolerance, not by round-off)."""
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cases", "variable3d_case.cpp")
    exe = build.compile_driver(src, str(tmp_path / "variable3d_case"))
    r = subprocess.run([exe, "solve"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("solution ")]
    z = load("dropin3d.npz")
    assert [row[1] for row in rows] == list(z["names"])
    got = np.array([[float(v) for v in row[2:]] for row in rows])
    np.testing.assert_allclose(got, z["values"], rtol=1e-9, atol=1e-11)
