"""Parity with the reference's own answer on a measured-size configuration: the cross of 5 x 1024^2 cells
with Neumann arm tips and a zero-mean Gaussian right-hand side (the headline workload's geometry at half
its side length), solved by the reference's own sources (oracle/_ref, ~15 s on 16 host threads) and by
every GPU form through the C ABI.

"The reference's answer" is its ConcatPoissonSolver2D::solve (GMRES tol 1e-14) refined once by the same
solver (oracle/refsolve.py): its plain FP64 answer carries round-off of about eps * cond(A), 3e-11 here, so
the refined one is what tighter forms are compared with, and the plain one is checked within its own
distance from it."""
import numpy as np
import pytest

from gpu_util import torch_cuda
from focalors_poisson_b200 import capi
from focalors_poisson_b200 import workloads as W
from oracle import refbind as R
from oracle import refsolve as RS

pytestmark = pytest.mark.gpu

N = 1024
SEED = 2024


@pytest.fixture(scope="module")
def case():
    assert R.available(), "oracle/_ref/libfpref.so (the reference's own sources, built by build()) is missing"
    g = W.cross(N, neumann_tips=True)
    rhs = W.gaussian_rhs(g, SEED)
    ref = RS.reference_answer(g, rhs)
    return g, rhs, ref


def _gpu(solver, rhs, fn):
    torch = torch_cuda()
    t = [torch.tensor(r, device="cuda") for r in rhs]
    info = fn(solver, t)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in t], info


FORMS = {
    # form: (how to run it, bound on rel L2 against the refined reference answer)
    "f64": (lambda s, t: s.solve(t), 1e-10),  # one FP64 solve: its own eps * cond round-off
    "f64ir": (lambda s, t: s.solve_ir(t, rel_tol=1e-13, max_refine=10, inner="f64"), 1e-12),
    "f32ir": (lambda s, t: s.solve_ir(t, rel_tol=1e-13, max_refine=10, inner="f32"), 1e-12),
    "mixedir": (lambda s, t: s.solve_ir(t, rel_tol=1e-13, max_refine=10, inner="mixed"), 1e-12),
}


def test_reference_answer_is_converged(case):
    """The refinement step changes the reference's answer by its round-off only, and leaves a residual at
    FP64 round-off: the refined answer is the discrete solution to ~1e-13."""
    g, rhs, ref = case
    assert ref["rel_residual"] < 1e-10 and ref["rel_correction"] < 1e-9, ref
    r = RS.residual(g, rhs, ref["refined"])
    fs = [f * h * h for f, h in zip(rhs, g.hx)]
    rel_res = float(np.sqrt(sum((x * x).sum() for x in r)) / np.sqrt(sum((x * x).sum() for x in fs)))
    assert rel_res < 1e-13, rel_res


@pytest.mark.parametrize("form", list(FORMS))
def test_spectral_forms_match_reference(case, form):
    g, rhs, ref = case
    fn, bound = FORMS[form]
    solver = capi.Composite(g, 20, 1e-14, 100)
    got, info = _gpu(solver, rhs, fn)
    err = RS.rel_l2(got, ref["refined"])
    plain = RS.rel_l2(got, ref["plain"])
    assert err <= bound, (form, err, info)
    # against the reference's plain answer: within that answer's own distance from the converged one
    assert plain <= max(bound, 3.0 * ref["rel_correction"]), (form, plain, ref["rel_correction"])


def test_schur_gmres_path_matches_reference(case):
    """The general path (interface-preconditioned Schur GMRES, the reference's algorithm on interface
    unknowns) on the same workload, GMRES tol 1e-14 as the reference."""
    g, rhs, ref = case
    solver = capi.Composite(g, 20, 1e-14, 100, spectral=False)
    got, info = _gpu(solver, rhs, lambda s, t: s.solve(t))
    assert info["converged"], info
    assert RS.rel_l2(got, ref["refined"]) <= 1e-10
    assert RS.rel_l2(got, ref["plain"]) <= max(1e-10, 3.0 * ref["rel_correction"])


@pytest.fixture(scope="module")
def tree_case():
    """The 9-subdomain tree of the large composite workload (centre, 4 arms, 4 corners on the N / S arms,
    W / E arms periodic in y, Neumann tip faces) at 128^2 per subdomain with its 32-bump right-hand side.
    Its depth-2 tree makes the reference build the Schur matrices of the internal arms itself, one subtree
    solve per interface cell (about a minute on 16 host threads at this size)."""
    assert R.available(), "oracle/_ref/libfpref.so (the reference's own sources, built by build()) is missing"
    g = W.tree9_large(128)
    rhs = W.gaussian_bumps_rhs(g, 5)
    return g, rhs, RS.reference_answer(g, rhs, 20, 1e-12, 100)


@pytest.mark.parametrize("form", ["f64", "f32ir"])
def test_large_tree_matches_reference(tree_case, form):
    """Root Schur GMRES with the internal children's Schur matrices from batched spectral subtree solves
    (FP64), and FP32-transform inner solves in FP64 refinement, against the reference's refined answer."""
    g, rhs, ref = tree_case
    solver = capi.Composite(g, 20, 1e-14, 200)
    if form == "f64":
        got, info = _gpu(solver, rhs, lambda s, t: s.solve(t))
        bound = 1e-10
    else:
        got, info = _gpu(solver, rhs, lambda s, t: s.solve_ir(t, rel_tol=1e-13, max_refine=10))
        bound = 1e-12
    err = RS.rel_l2(got, ref["refined"])
    assert err <= bound, (form, err, info)
    assert RS.rel_l2(got, ref["plain"]) <= max(bound, 3.0 * ref["rel_correction"])
