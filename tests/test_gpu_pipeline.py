"""Pipelined host-buffer solves (fp_composite_solve_async / fp_composite_wait) against the synchronous
host-pointer solves of the same forms, and the refinement graph (the correction loop as a CUDA graph while
node) against the reference's own answers."""
import types

import numpy as np
import pytest

from golden_io import composite_case, rel_l2, tight_outputs
from gpu_util import torch_cuda
from focalors_poisson_b200 import capi
from focalors_poisson_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORMS = ["f64", "f64ir", "f32ir", "mixedir"]
INNER = {"f64ir": "f64", "f32ir": "f32", "mixedir": "mixed"}


def _sync(solver, rhs, form, ghosts=None, rel_tol=1e-12, max_refine=10):
    f = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    if form == "f64":
        info = solver.solve(f, ghosts)
    else:
        info = solver.solve_ir(f, ghosts, rel_tol=rel_tol, max_refine=max_refine, inner=INNER[form])
    return f, info


def _pinned(arrays):
    torch = torch_cuda()
    return [torch.tensor(np.asarray(a), dtype=torch.float64).pin_memory() for a in arrays]


@pytest.fixture(scope="module")
def cross():
    g = W.cross(128, neumann_tips=True)
    return g, capi.Composite(g, 20, 1e-14, 100), W.gaussian_rhs(g, 11)


@pytest.mark.parametrize("form", FORMS)
def test_async_matches_sync(cross, form):
    """One queued solve per form equals the synchronous host-pointer solve of the same form, and the info
    reports the same refinement steps."""
    g, solver, rhs = cross
    want, winfo = _sync(solver, rhs, form)
    out = [np.zeros_like(r) for r in rhs]
    solver.solve_async(rhs, out, form=form, rel_tol=1e-12, max_refine=10)
    info = solver.wait()
    assert rel_l2(out, want) <= 1e-14, form
    assert info["refinements"] == winfo["refinements"], (info, winfo)


def test_async_queue_of_distinct_problems(cross):
    """Several calls queued before one wait, each with its own right-hand sides (page-locked) and outputs:
    every output is its own problem's solution."""
    g, solver, _ = cross
    rhss = [W.gaussian_rhs(g, 100 + k) for k in range(5)]
    ins = [_pinned(r) for r in rhss]
    outs = [_pinned([np.zeros_like(a) for a in r]) for r in rhss]
    for i, o in zip(ins, outs):
        solver.solve_async(i, o, form="mixedir", rel_tol=1e-12, max_refine=10)
    solver.wait(check_convergence=True)
    for r, o in zip(rhss, outs):
        want, _ = _sync(solver, r, "mixedir")
        assert rel_l2([x.numpy() for x in o], want) <= 1e-14


def test_async_in_place_chain(cross):
    """out == rhs, and the next call reads the previous call's output as its right-hand side: the second
    result is A^-1 (A^-1 b), as two synchronous solves give."""
    g, solver, rhs = cross
    buf = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    solver.solve_async(buf, buf, form="f64")
    solver.solve_async(buf, buf, form="f64")
    solver.wait()
    once, _ = _sync(solver, rhs, "f64")
    twice, _ = _sync(solver, once, "f64")
    assert rel_l2(buf, twice) <= 1e-14


@pytest.mark.parametrize("name", ["cross24_ghosts.npz", "lt_shape_1.npz"])
def test_async_ghosts_and_reference(name):
    """Ghost buffers travel with the call; the refined answer matches the reference's own output."""
    geo, rhs, ghosts, outs, (m, tol, it), root = composite_case(name)
    solver = capi.Composite(types.SimpleNamespace(**geo), m, tol, it, root=root)
    out = [np.zeros_like(np.asarray(r, dtype=np.float64)) for r in rhs]
    ins = [np.array(r, dtype=np.float64, copy=True) for r in rhs]
    solver.solve_async(ins, out, ghosts=ghosts, form="mixedir", rel_tol=1e-13, max_refine=10)
    solver.wait()
    want, _ = _sync(solver, rhs, "mixedir", ghosts, rel_tol=1e-13)
    assert rel_l2(out, want) <= 1e-14
    assert rel_l2(out, tight_outputs(name)) <= 1e-10, name


def test_async_schur_path(cross):
    """Outside the spectral path (FP_NO_SPECTRAL) the queued solve runs the Schur GMRES and still matches."""
    g, _, rhs = cross
    solver = capi.Composite(g, 20, 1e-12, 100, spectral=False)
    want, _ = _sync(solver, rhs, "f64")
    out = [np.zeros_like(r) for r in rhs]
    solver.solve_async(rhs, out, form="f64")
    info = solver.wait(check_convergence=True)
    assert info["converged"]
    assert rel_l2(out, want) <= 1e-14


def test_async_errors_and_empty_wait(cross):
    g, solver, rhs = cross
    solver.wait()  # nothing queued
    out = [np.zeros_like(r) for r in rhs]
    with pytest.raises(ValueError):
        solver.solve_async(rhs, out, form="f16")
    with pytest.raises(capi.FpError):
        solver.solve_async(rhs, out, form="f32ir", rel_tol=-1.0)
    solver.wait()


def test_refinement_graph_steps_bounded(cross):
    """A tolerance below round-off makes the device-side stop rule end the graph's loop at max_refine."""
    g, solver, rhs = cross
    for k in (2, 3, 5):
        f, info = _sync(solver, rhs, "f32ir", rel_tol=1e-30, max_refine=k)
        assert info["refinements"] == k
        assert np.isfinite(np.concatenate([x.ravel() for x in f])).all()
