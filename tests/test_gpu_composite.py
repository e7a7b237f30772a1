"""GPU parity of the composite (ConcatPoissonSolver2D) solve against the reference's own outputs
(tests/golden/*.npz, generated from its sources) through the C ABI."""
import types

import numpy as np
import pytest

from golden_io import COMPOSITE_CASES, composite_case, rel_l2, tight_outputs
from gpu_util import torch_cuda
from focalors_poisson_b200 import capi
from focalors_poisson_b200 import workloads as W

pytestmark = pytest.mark.gpu


def geometry(geo):
    return types.SimpleNamespace(**geo)


@pytest.mark.parametrize("name", COMPOSITE_CASES)
def test_composite_golden_fullfield(name):
    """Full-field Krylov vectors follow the reference's own iterates: agreement to 1e-12 at the case's tol."""
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    solver = capi.Composite(geometry(geo), m, tol, it, root=root, fullfield=True)
    assert solver.tree()[0] == root
    fields = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    info = solver.solve(fields, ghosts)
    assert info["converged"]
    assert rel_l2(fields, outs) <= 1e-12, name


@pytest.mark.parametrize("name", COMPOSITE_CASES)
@pytest.mark.parametrize("inverse", [True, False])
def test_composite_golden_interface(name, inverse):
    """Interface Krylov vectors (the default) converge along a different path under the reference's own
    full-field stopping test. Driven to tol 1e-15 they agree with the reference driven to 1e-15 within
    1e-12; at the case's tol they stay within the reference's own distance from that converged answer."""
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    tight = tight_outputs(name)
    own_err = rel_l2(outs, tight)
    solver = capi.Composite(geometry(geo), m, 1e-15, it, root=root, interface_inverse=inverse)
    fields = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    solver.solve(fields, ghosts)  # 1e-15 is below the round-off floor of some cases: both stop at max_iter
    assert rel_l2(fields, tight) <= 1e-12, name
    solver.set_parameter(m, tol, it)
    fields = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    assert solver.solve(fields, ghosts)["converged"]
    assert rel_l2(fields, outs) <= max(1e-12, 3.0 * own_err), (name, own_err)


def test_composite_device_pointers_and_repeat():
    torch = torch_cuda()
    name = "cross48_neumann_tips.npz"
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    own_err = rel_l2(outs, tight_outputs(name))
    solver = capi.Composite(geometry(geo), m, tol, it, root=root)
    results = []
    for _ in range(2):  # solve() consumes its inputs: re-fill and solve again, same answer
        t = [torch.tensor(r, device="cuda") for r in rhs]
        solver.solve(t)
        torch.cuda.synchronize()
        results.append([x.cpu().numpy() for x in t])
    assert rel_l2(results[0], outs) <= max(1e-12, 3.0 * own_err)
    for a, b in zip(*results):
        np.testing.assert_array_equal(a, b)


def test_root_choice_matches_reference_rule():
    g = W.tree9(8)
    solver = capi.Composite(g, 20, 1e-12, 100)
    root, lv = solver.tree()
    assert root == 0 and list(lv) == [0, 1, 1, 1, 1, 2, 2, 2, 2]


def test_cyclic_geometry_rejected():
    # 2x2 block grid: A-B, A-C, B-D, C-D is a cycle the reference's tree builder cannot hold
    n = 8
    geo = types.SimpleNamespace(nx=[n] * 4, ny=[n] * 4, hx=[0.1] * 4, hy=[0.1] * 4, bc=[[0] * 4] * 4,
                                connections=[(0, 1, 1), (0, 3, 2), (1, 3, 3), (2, 1, 3)])
    with pytest.raises(capi.FpError) as e:
        capi.Composite(geo)
    assert e.value.code == 1 and "cycle" in str(e.value)


@pytest.mark.parametrize("name", COMPOSITE_CASES)
def test_composite_f32_refinement(name):
    """FP32-transform inner solves + FP64 iterative refinement reach the reference's converged answer to
    1e-10 relative L2 (the target of the reduced-precision form)."""
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    tight = tight_outputs(name)
    solver = capi.Composite(geometry(geo), m, tol, it, root=root)
    fields = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    info = solver.solve_ir(fields, ghosts, rel_tol=1e-12, max_refine=8)
    assert info["refinements"] >= 2, info
    assert rel_l2(fields, tight) <= 1e-10, (name, info, rel_l2(fields, tight))


@pytest.mark.parametrize("name", ["cross48_neumann_tips.npz", "cross24_ghosts.npz", "tree9_periodic.npz"])
def test_composite_residual_of_reference_solution(name):
    """The composite 5-point operator behind fp_composite_residual is the one the reference inverts: its
    converged solutions have relative residual at round-off, a perturbed one does not."""
    torch = torch_cuda()
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    tight = tight_outputs(name)
    solver = capi.Composite(geometry(geo), m, tol, it, root=root)
    u = [torch.tensor(t, device="cuda") for t in tight]
    f = [torch.tensor(r, device="cuda") for r in rhs]
    g = None if ghosts is None else [[None if x is None else torch.tensor(x, device="cuda") for x in row]
                                     for row in ghosts]
    assert solver.residual(u, f, g) <= 1e-11
    u[0][1, 1] += 1e-3 * float(u[0].abs().max())
    assert solver.residual(u, f, g) > 1e-6


@pytest.mark.parametrize("n", [256, 1024])
def test_spectral_path_matches_schur_gmres(n):
    """A cross with Neumann arm tips is inside the spectral path's scope: its direct solve equals the Schur
    GMRES driven to tol 1e-14 (FP_NO_SPECTRAL), and its FP32 refinement reaches the same answer."""
    torch = torch_cuda()
    g = W.cross(n, neumann_tips=True)
    rhs = W.gaussian_rhs(g, 31)
    spec = capi.Composite(g, 20, 1e-12, 100)
    gm = capi.Composite(g, 20, 1e-14, 200, spectral=False)
    a = [torch.tensor(r, device="cuda") for r in rhs]
    b = [x.clone() for x in a]
    c = [x.clone() for x in a]
    d = [x.clone() for x in a]
    info = spec.solve(a)
    assert info["converged"] and info["iterations"] == 0  # no Krylov iteration on the spectral path
    gm.solve(b)
    spec.solve_ir(c, rel_tol=1e-13, max_refine=8)
    mixed = spec.solve_ir(d, rel_tol=1e-13, max_refine=8, inner="mixed")
    torch.cuda.synchronize()
    got, want, ir, mx = ([x.cpu().numpy() for x in v] for v in (a, b, c, d))
    # every FP64 answer carries round-off of order eps * cond(A) (~5e-11 at 1024^2)
    tol = 1e-11 if n <= 256 else 1e-10
    assert rel_l2(got, want) <= tol, rel_l2(got, want)
    assert rel_l2(ir, want) <= tol, rel_l2(ir, want)
    assert rel_l2(mx, want) <= tol, rel_l2(mx, want)
    assert rel_l2(mx, ir) <= 1e-11 and mixed["refinements"] <= 3, (rel_l2(mx, ir), mixed)


def test_large_tree_spectral_schur_construction():
    """The 9-subdomain tree with periodic arms (depth 2): the Schur matrices of its internal children are
    built from batched spectral subtree solves; the result equals the full-field GMRES with the nested
    impulse construction (the reference's), and its residual is at round-off."""
    torch = torch_cuda()
    g = W.tree9_large(64)
    rhs = W.gaussian_bumps_rhs(g, 5)
    fast = capi.Composite(g, 20, 1e-14, 300)
    ref = capi.Composite(g, 20, 1e-14, 300, fullfield=True)
    a = [torch.tensor(r, device="cuda") for r in rhs]
    b = [x.clone() for x in a]
    pristine = [x.clone() for x in a]
    fast.solve(a)
    ref.solve(b)
    torch.cuda.synchronize()
    got, want = [x.cpu().numpy() for x in a], [x.cpu().numpy() for x in b]
    assert rel_l2(got, want) <= 1e-10, rel_l2(got, want)
    assert fast.residual(a, pristine) <= 1e-10

