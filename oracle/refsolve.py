"""The reference's own composite solve at large sizes, with one refinement step by the same solver.

TEST AND CPU-BASELINE INFRASTRUCTURE. Callers: tests/ (parity of the GPU path against the reference on
the measured configurations) and bench.py's CPU legs. Nothing in the product imports it.

`reference_answer(g, rhs)` runs ConcatPoissonSolver2D::solve (pe/concat/concat_solver2d.cpp:101-157) of
the reference's own sources (oracle/_ref) on the geometry `g` (a focalors_poisson_b200.workloads.Geometry)
and returns its answer. The root Schur matrices are injected in closed form (oracle/schur_closed_form.py,
checked against the reference's own impulse construction to round-off), because that construction takes one
full solve per interface cell, hours at 2048^2.

A single FP64 solve of the reference carries its own round-off, about eps * cond(A) (3e-11 relative L2 on
the 5 x 1024^2 Neumann-tip cross, more at 2048^2). To compare answers below that level, the reference's
answer is refined once with the reference's own solver: r = fs - A u (fs the hx^2-scaled right-hand side,
A the composite 5-point operator of oracle/fp_oracle.py composite_apply, in extended precision), then
u + solve(r / hx^2), with r scaled to the right-hand side's norm for that solve because the reference's GMRES
tolerance is absolute.
Both the plain and the refined answer are returned; "the reference's solution" in the parity tests is the
refined one, and the plain one is reported beside it.
"""
from __future__ import annotations

import numpy as np

from . import fp_oracle as O
from . import refbind as R
from . import schur_closed_form as SC


def _norm(fields):
    return float(np.sqrt(sum(float((x * x).sum()) for x in fields)))


def reference_case(g, m: int = 20, tol: float = 1e-14, max_iter: int = 100):
    """The reference's solver object for geometry g (outer faces only carry boundary codes; the reference
    marks the connected faces Adjacented itself). When every child of the root is a leaf its Schur matrices
    are injected in closed form; deeper trees (a child with children of its own) are constructed by the
    reference itself, one subtree solve per interface cell, which is practical at a few hundred cells a
    side."""
    lx = [a * h for a, h in zip(g.nx, g.hx)]
    ly = [b * h for b, h in zip(g.ny, g.hy)]
    bco = [[0 if b == 3 else b for b in row] for row in g.bc]
    try:
        schur = SC.root_schur_matrices(g)
    except ValueError:
        schur = None
    return R.ConcatCase(g.nx, g.ny, lx, ly, g.connections, bco, m, tol, max_iter, schur=schur)


def residual(g, rhs, u):
    """fs - A u in the hx^2-scaled form the reference solves (zero ghost buffers), evaluated in extended
    precision (numpy longdouble) and rounded to FP64 once: for smooth solutions the stencil's terms are
    ~cond(A) times larger than the residual, and a plain FP64 evaluation would carry ~eps * cond(A) of
    round-off, more than the answers it is meant to separate."""
    doms = [O.Domain(a, b, h1, h2, [0 if x == 3 else x for x in bcs])
            for a, b, h1, h2, bcs in zip(g.nx, g.ny, g.hx, g.hy, g.bc)]
    ul = [np.asarray(x, dtype=np.longdouble) for x in u]
    au = O.composite_apply(doms, g.connections, g.bc, ul)
    h2 = [np.longdouble(h) * np.longdouble(h) for h in g.hx]
    return [np.asarray(np.asarray(f, dtype=np.longdouble) * s - a, dtype=np.float64) for f, s, a in zip(rhs, h2, au)]


def reference_answer(g, rhs, m: int = 20, tol: float = 1e-14, max_iter: int = 100, refine: bool = True,
                     case=None):
    """{"plain": u, "refined": u + e, "seconds": solve time, "refine_seconds", "rel_residual" (of the plain
    answer), "rel_correction" (|e| / |u|)}. Right-hand sides are not modified."""
    case = case or reference_case(g, m, tol, max_iter)
    u, t = case.solve([np.array(r, dtype=np.float64, copy=True) for r in rhs])
    out = {"plain": u, "seconds": t}
    if not refine:
        return out
    r = residual(g, rhs, u)
    fs_norm = _norm([f * h * h for f, h in zip(rhs, g.hx)])
    # the reference's GMRES tolerance is absolute: the residual is scaled up to the right-hand side's norm
    # (the problem is linear) so that the correction is solved to the same relative accuracy as u
    sc = fs_norm / max(_norm(r), 1e-300)
    e, t2 = case.solve([x * (sc / (h * h)) for x, h in zip(r, g.hx)])
    e = [x / sc for x in e]
    out.update({"refined": [a + b for a, b in zip(u, e)], "refine_seconds": t2,
                "rel_residual": _norm(r) / fs_norm, "rel_correction": _norm(e) / _norm(u)})
    return out


def rel_l2(a, b) -> float:
    """Relative L2 distance of field lists a and b over all cells, relative to b."""
    num = sum(float(((np.asarray(x) - np.asarray(y)) ** 2).sum()) for x, y in zip(a, b))
    return float(np.sqrt(num) / _norm([np.asarray(y) for y in b]))
