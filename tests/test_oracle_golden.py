"""Pins the oracle (oracle/fp_oracle.py, a numpy restatement of the reference) against golden vectors
produced by the reference's own C++ sources (tests/golden/make_golden.py). CPU only."""
import numpy as np
import pytest

from golden_io import COMPOSITE_CASES, CONCAT3D_CASES, composite_case, concat3d_case, load, rel_l2
from oracle import fp_oracle as O

KINDS = ["DD", "NN", "ND", "DN", "PP"]


def test_transforms_match_reference():
    z = load("transforms.npz")
    seen = 0
    for key in z.files:
        if not key.startswith("in_"):
            continue
        _, kind, ny = key.split("_")
        f = z[key]
        for tag, fn in (("fwd", O.transform_forward), ("inv", O.transform_inverse)):
            ref = z[f"{tag}_{kind}_{ny}"]
            got = fn(kind, f)
            assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max()), (kind, ny, tag)
            seen += 1
    assert seen >= 100


def test_poisson_reference_driver_fixture():
    """case/validation/2d/poisson_solver_reference.cpp: 3x4, hx=1, hy=2, 25 boundary combinations."""
    z = load("poisson.npz")
    f = np.arange(12, dtype=np.float64).reshape(3, 4) + 1.0
    for c, bc in enumerate(z["combos"]):
        got = O.PoissonSolver2D(3, 4, 1.0, 2.0, [int(b) for b in bc]).solve(f)
        ref = z[f"fixture_{c}"]
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (c, bc)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_poisson_random(tag):
    z = load("poisson.npz")
    f = z[f"rand_{tag}_in"]
    nx, ny, hx, hy = z[f"rand_{tag}_shape"]
    n = 0
    for c, bc in enumerate(z["combos"]):
        key = f"rand_{tag}_{c}"
        if key not in z.files:
            continue
        got = O.PoissonSolver2D(int(nx), int(ny), hx, hy, [int(b) for b in bc]).solve(f)
        ref = z[key]
        assert np.abs(got - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), (tag, c, bc)
        n += 1
    assert n >= 20


@pytest.mark.parametrize("name", COMPOSITE_CASES)
def test_composite_matches_reference(name):
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    doms = [O.Domain(a, b, hx, hy, bc) for a, b, hx, hy, bc in zip(geo["nx"], geo["ny"], geo["hx"], geo["hy"],
                                                                   geo["bc"])]
    for d in doms:
        d.bc = [O.D if b == O.ADJ else b for b in d.bc]
    s = O.ConcatPoissonSolver2D(doms, geo["connections"], m, tol, it, root=root)
    assert s.tree.root == root
    got = s.solve(rhs, ghosts)
    assert rel_l2(got, outs) <= 1e-12, name


def test_mock_fixtures():
    """gmres_reference.cpp / shur_mat_reference.cpp with the mock branch solver."""
    z = load("mocks.npz")
    for loc in range(4):
        nbx, nby = (4, 5) if loc in (0, 1) else (3, 4)
        g = O.GMRESSolver2D(2, 1e-3, 2, O.mock_solve)
        g.S = [(loc, O.schur_matrix(loc, nbx, nby, O.mock_solve))]
        got = g.solve(np.arange(15, dtype=np.float64).reshape(3, 5) + 1.0)
        ref = z[f"gmres_{loc}"]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    dims = [(6, 3, 4, 3), (6, 3, 4, 3), (3, 6, 3, 4), (3, 6, 3, 4)]
    for loc, (bnx, bny, nx, ny) in enumerate(dims):
        S = O.schur_matrix(loc, bnx, bny, O.mock_solve)
        np.testing.assert_array_equal(S, z[f"schur_S_{loc}"])
        f = np.arange(nx * ny, dtype=np.float64).reshape(nx, ny) + 1.0
        np.testing.assert_array_equal(O.schur_apply(loc, S, f), z[f"schur_prod_{loc}"])


def test_poisson3d_matches_reference():
    """The 3D rectangle solve (PoissonSolver3D) restated in numpy against the reference's own output: 100
    boundary combinations on 6 x 6 x 4 cells and two cases of 64 cells along x."""
    z = load("poisson3d.npz")
    f = z["small_in"]
    for c, bc in enumerate(z["combos"]):
        got = O.PoissonSolver3D(6, 6, 4, 0.3, 0.2, 0.25, [int(b) for b in bc]).solve(f)
        ref = z[f"small_{c}"]
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (c, bc)
    for tag in ("a", "b"):
        g = z[f"{tag}_in"]
        got = O.PoissonSolver3D(*g.shape, *z[f"{tag}_h"], [int(b) for b in z[f"{tag}_bc"]]).solve(g)
        ref = z[f"{tag}_out"]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), tag


@pytest.mark.parametrize("name", CONCAT3D_CASES)
def test_concat3d_matches_reference(name):
    """The oracle's ConcatPoissonSolver3D (tree, Schur matrices by impulse solves, GMRES on full fields, the
    two passes) against the reference's own solve of the same case: same tree, same answer to round-off."""
    doms, conns, bc, rhs, ghosts, outs, tight, root, levels = concat3d_case(name)
    D3 = [O.Domain3(*d, list(b)) for d, b in zip(doms, bc)]
    s = O.ConcatPoissonSolver3D(D3, conns, 20, 1e-12, 100)
    assert s.tree.root == root
    for lv, members in enumerate(s.tree.levels):
        assert all(levels[d] == lv for d in members)
    got = s.solve(rhs, ghosts)
    assert rel_l2(got, outs) <= 1e-13, name

