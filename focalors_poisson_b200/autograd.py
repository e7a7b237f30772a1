"""Differentiable composite solve: torch.autograd.Function over the GPU forward and adjoint solves.

    u = solve(solver, rhs, scale=None, ghosts=None, form="f32ir")

solves the composite problem of `solver` (a capi.Composite) for the right-hand side `scale * rhs` (per-cell
source scale, optional) with fixed ghost buffers, and returns one tensor per domain. Backward runs the
hand-written transposed solve (capi.Composite.adjoint / adjoint_ir, fp_composite_adjoint_* in
include/fp_capi.h) once for all domains:

    g = H A^-1 (dL/du),   dL/drhs = scale * g,   dL/dscale = rhs * g

with H = diag(hx^2) and A the composite operator ConcatPoissonSolver2D::solve inverts
(pe/concat/concat_solver2d.cpp:101-157). Forms: "f64" (one FP64 solve per call), "f32ir" (FP32 transforms
in FP64 iterative refinement to rel_tol), "f64ir" (FP64 solves in FP64 refinement). Tensors must be CUDA
float64 fields of the domains' shapes; there is no CPU path.
"""
from __future__ import annotations

import torch

from . import capi

FORMS = ("f64", "f32ir", "f64ir")


def _forward(solver, fields, ghosts, form, rel_tol, max_refine):
    if form == "f64":
        return solver.solve(fields, ghosts)
    return solver.solve_ir(fields, ghosts, rel_tol=rel_tol, max_refine=max_refine,
                           inner="f32" if form == "f32ir" else "f64")


def _adjoint(solver, fields, form, rel_tol, max_refine):
    if form == "f64":
        return solver.adjoint(fields)
    return solver.adjoint_ir(fields, rel_tol=rel_tol, max_refine=max_refine, inner="f32" if form == "f32ir" else "f64")


class CompositeSolve(torch.autograd.Function):
    """apply(solver, ghosts, form, rel_tol, max_refine, nd, has_scale, *rhs, *scale) -> tuple of nd fields."""

    @staticmethod
    def forward(ctx, solver, ghosts, form, rel_tol, max_refine, nd, has_scale, *tensors):
        rhs = tensors[:nd]
        scale = tensors[nd:2 * nd] if has_scale else None
        for t in tensors:
            if not (t.is_cuda and t.dtype == torch.float64):
                raise TypeError("the composite solve takes CUDA float64 tensors")
        u = [(r * s if has_scale else r).contiguous().clone() for r, s in zip(rhs, scale or rhs)]
        ctx.info = _forward(solver, u, ghosts, form, rel_tol, max_refine)
        ctx.solver, ctx.form, ctx.rel_tol, ctx.max_refine, ctx.nd, ctx.has_scale = (
            solver, form, rel_tol, max_refine, nd, has_scale)
        ctx.save_for_backward(*tensors)
        return tuple(u)

    @staticmethod
    def backward(ctx, *grad_u):
        nd = ctx.nd
        saved = ctx.saved_tensors
        rhs = saved[:nd]
        scale = saved[nd:2 * nd] if ctx.has_scale else None
        g = [(gu if gu is not None else torch.zeros_like(r)).to(torch.float64).contiguous().clone()
             for gu, r in zip(grad_u, rhs)]
        ctx.adjoint_info = _adjoint(ctx.solver, g, ctx.form, ctx.rel_tol, ctx.max_refine)
        grad_rhs = [gi * s for gi, s in zip(g, scale)] if ctx.has_scale else g
        grads = list(grad_rhs)
        if ctx.has_scale:
            grads += [gi * r for gi, r in zip(g, rhs)]
        return (None,) * 7 + tuple(grads)


def solve(solver: "capi.Composite", rhs, scale=None, ghosts=None, form: str = "f32ir", rel_tol: float = 1e-12,
          max_refine: int = 10):
    """Differentiable composite solve; returns a list of solution tensors (one per domain)."""
    if form not in FORMS:
        raise ValueError(f"form must be one of {FORMS}")
    rhs = list(rhs)
    nd = len(rhs)
    has_scale = scale is not None
    tensors = rhs + (list(scale) if has_scale else [])
    return list(CompositeSolve.apply(solver, ghosts, form, float(rel_tol), int(max_refine), nd, has_scale, *tensors))
