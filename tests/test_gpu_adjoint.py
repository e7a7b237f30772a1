"""GPU adjoint solve (fp_composite_adjoint_*) and the differentiable solve (focalors_poisson_b200.autograd):
dot-product tests of the transposed solve, gradients against the FP64 oracle's gradient, and the
differentiable cross workload (5 x 512^2, FP32 transforms + FP64 refinement) against central finite
differences with step 1e-4 on 64 random entries of the right-hand side and of the source scale."""
import types

import numpy as np
import pytest

from adjoint_cases import CASES
from golden_io import COMPOSITE_CASES, composite_case
from gpu_util import torch_cuda
from focalors_poisson_b200 import autograd as FA
from focalors_poisson_b200 import capi
from focalors_poisson_b200 import workloads as W
from oracle import fp_oracle as O
from oracle import schur_closed_form as SC

pytestmark = pytest.mark.gpu


def _dot(a, b):
    return sum(float((x * y).sum()) for x, y in zip(a, b))


def _geometries():
    out = {k: v() for k, v in CASES.items()}
    for name in COMPOSITE_CASES:
        if "tight" in name:
            continue
        geo = composite_case(name)[0]
        out[name] = types.SimpleNamespace(**geo)
    return out


GEOS = _geometries()


@pytest.mark.parametrize("name", sorted(GEOS))
@pytest.mark.parametrize("form", ["f64", "f32ir"])
def test_adjoint_dot_product(name, form):
    """<solve(f), g> = <f, adjoint(g)> to round-off, zero ghosts (the map whose transpose is computed)."""
    torch = torch_cuda()
    geo = GEOS[name]
    solver = capi.Composite(geo, 20, 1e-14, 200)
    rng = np.random.default_rng(11)
    f = [torch.tensor(rng.standard_normal((a, b)), device="cuda") for a, b in zip(geo.nx, geo.ny)]
    g = [torch.tensor(rng.standard_normal((a, b)), device="cuda") for a, b in zip(geo.nx, geo.ny)]
    u, v = [x.clone() for x in f], [x.clone() for x in g]
    if not any(b == 0 for row in geo.bc for b in row):
        with pytest.raises(capi.FpError):
            solver.adjoint(v)
        return
    if form == "f64":
        solver.solve(u)
        solver.adjoint(v)
    else:
        solver.solve_ir(u, rel_tol=1e-13, max_refine=10)
        solver.adjoint_ir(v, rel_tol=1e-13, max_refine=10)
    torch.cuda.synchronize()
    lhs, rhs = _dot(u, g), _dot(f, v)
    scale = (_dot(u, u) * _dot(g, g)) ** 0.5
    assert abs(lhs - rhs) <= 1e-11 * scale, (name, lhs, rhs, scale)


def test_adjoint_host_pointers_match_device():
    torch = torch_cuda()
    geo = CASES["skewed_t"]()
    solver = capi.Composite(geo, 20, 1e-14, 200)
    rng = np.random.default_rng(3)
    g = [rng.standard_normal((a, b)) for a, b in zip(geo.nx, geo.ny)]
    host = [x.copy() for x in g]
    solver.adjoint(host)
    dev = [torch.tensor(x, device="cuda") for x in g]
    solver.adjoint(dev)
    torch.cuda.synchronize()
    for a, b in zip(host, dev):
        np.testing.assert_array_equal(a, b.cpu().numpy())


def _oracle_gradient(geo, f, s, ut, schur=None):
    """FP64 oracle: u = solve(s f); dL/df = s * H solve(H^-1 (u - u_t)), dL/ds = f * (the same)."""
    doms = [O.Domain(a, b, hx, hy, list(bc)) for a, b, hx, hy, bc in zip(geo.nx, geo.ny, geo.hx, geo.hy, geo.bc)]
    solver = O.ConcatPoissonSolver2D(doms, geo.connections, 20, 1e-13, 300, schur=schur)
    u = solver.solve([x * y for x, y in zip(f, s)])
    h2 = [hx * hx for hx in geo.hx]
    lam = solver.solve([(a - b) / c for a, b, c in zip(u, ut, h2)])
    lam = [x * c for x, c in zip(lam, h2)]
    return u, [x * y for x, y in zip(lam, s)], [x * y for x, y in zip(lam, f)]


def _reference_gradient(geo, f, s, ut):
    """The same FP64 gradient from the reference's own sources (oracle/_ref, the root Schur matrices in
    closed form) when that library was built, else from the numpy oracle (minutes at 512^2)."""
    from oracle import refbind as R

    S = SC.root_schur_matrices(geo)
    if not R.available():
        return _oracle_gradient(geo, f, s, ut, schur=S)
    lx = [a * h for a, h in zip(geo.nx, geo.hx)]
    ly = [b * h for b, h in zip(geo.ny, geo.hy)]
    bco = [[0 if b == 3 else b for b in row] for row in geo.bc]
    case = R.ConcatCase(geo.nx, geo.ny, lx, ly, geo.connections, bco, 20, 1e-15, 200, schur=S)
    u = case.solve([x * y for x, y in zip(f, s)])[0]
    h2 = [hx * hx for hx in geo.hx]
    lam = case.solve([(a - b) / c for a, b, c in zip(u, ut, h2)])[0]
    lam = [x * c for x, c in zip(lam, h2)]
    return u, [x * y for x, y in zip(lam, s)], [x * y for x, y in zip(lam, f)]


@pytest.mark.parametrize("name", ["skewed_t", "periodic_arm"])
@pytest.mark.parametrize("form", ["f64", "f32ir"])
def test_autograd_matches_oracle_gradient(name, form):
    torch = torch_cuda()
    geo = CASES[name]()
    rng = np.random.default_rng(5)
    f = [rng.standard_normal((a, b)) for a, b in zip(geo.nx, geo.ny)]
    s = [rng.uniform(0.5, 1.5, (a, b)) for a, b in zip(geo.nx, geo.ny)]
    ut = [rng.standard_normal((a, b)) for a, b in zip(geo.nx, geo.ny)]
    u_ref, gf_ref, gs_ref = _oracle_gradient(geo, f, s, ut)
    solver = capi.Composite(geo, 20, 1e-14, 200)
    ft = [torch.tensor(x, device="cuda", requires_grad=True) for x in f]
    st = [torch.tensor(x, device="cuda", requires_grad=True) for x in s]
    utt = [torch.tensor(x, device="cuda") for x in ut]
    u = FA.solve(solver, ft, st, form=form, rel_tol=1e-13)
    loss = 0.5 * sum(((a - b) ** 2).sum() for a, b in zip(u, utt))
    loss.backward()
    rel = lambda a, b: (_dot([x - y for x, y in zip(a, b)], [x - y for x, y in zip(a, b)]) / _dot(b, b)) ** 0.5
    assert rel([x.detach().cpu().numpy() for x in u], u_ref) <= 1e-11
    assert rel([x.grad.cpu().numpy() for x in ft], gf_ref) <= 1e-11
    assert rel([x.grad.cpu().numpy() for x in st], gs_ref) <= 1e-11


def test_differentiable_cross_512_finite_differences():
    """The differentiable cross workload: 5 x 512^2, FP32 transforms + FP64 refinement. Gradients with
    respect to the RHS and the source scale against (1) the FP64 oracle's gradient (closed-form root
    Schur matrices, oracle/schur_closed_form.py) and (2) central finite differences of the loss, step
    1e-4, on 64 random entries each. The loss difference of a probe pair is evaluated as
    sum((u+ - u-) * ((u+ + u-)/2 - u_t)), the exact algebraic form of 0.5|u+ - u_t|^2 - 0.5|u- - u_t|^2
    that avoids cancelling two O(1e5) sums."""
    torch = torch_cuda()
    g, f, s, ut, probes = W.adjoint_case(512)
    solver = capi.Composite(g, 20, 1e-14, 100)
    ft = [torch.tensor(x, device="cuda", requires_grad=True) for x in f]
    st = [torch.tensor(x, device="cuda", requires_grad=True) for x in s]
    utt = [torch.tensor(x, device="cuda") for x in ut]
    u = FA.solve(solver, ft, st, form="f32ir", rel_tol=1e-13)
    loss = 0.5 * sum(((a - b) ** 2).sum() for a, b in zip(u, utt))
    loss.backward()
    gf = [x.grad.detach() for x in ft]
    gs = [x.grad.detach() for x in st]

    # (1) FP64 oracle gradient
    u_ref, gf_ref, gs_ref = _reference_gradient(g, f, s, ut)
    rel = lambda a, b: (_dot([x - y for x, y in zip(a, b)], [x - y for x, y in zip(a, b)]) / _dot(b, b)) ** 0.5
    assert rel([x.cpu().numpy() for x in gf], gf_ref) <= 1e-10
    assert rel([x.cpu().numpy() for x in gs], gs_ref) <= 1e-10

    # (2) central finite differences
    step = 1e-4
    base = [torch.tensor(x * y, device="cuda") for x, y in zip(f, s)]

    def solve_eff(eff):
        w = [x.clone() for x in eff]
        solver.solve_ir(w, rel_tol=1e-13, max_refine=10)
        return w

    errs = []
    for which in ("rhs", "scale"):
        for d, i, j in probes:
            # perturbing f[d][i,j] by +-h changes the effective RHS by +-h s; perturbing s by +-h, by +-h f
            delta = step * (s[d][i, j] if which == "rhs" else f[d][i, j])
            plus = [x.clone() for x in base]
            minus = [x.clone() for x in base]
            plus[d][i, j] += delta
            minus[d][i, j] -= delta
            up, um = solve_eff(plus), solve_eff(minus)
            dl = sum(float(((a - b) * (0.5 * (a + b) - t)).sum()) for a, b, t in zip(up, um, utt))
            fd = dl / (2 * step)
            ad = float((gf if which == "rhs" else gs)[d][i, j])
            errs.append((abs(fd - ad), abs(ad), which, (d, i, j)))
    worst = max(errs, key=lambda e: e[0] / max(e[1], 1e-300))
    gmax = max(e[1] for e in errs)
    print(f"FD check: max |fd - ad| = {max(e[0] for e in errs):.3e}, max |ad| = {gmax:.3e}, "
          f"worst relative {worst[0] / max(worst[1], 1e-300):.3e} at {worst[2:]}")
    # bound relative to the gradient's scale over the probes: single entries can be far below it, where the
    # finite difference itself only resolves ~1e-11 (round-off of the two perturbed solves)
    assert max(e[0] for e in errs) <= 1e-6 * gmax, worst
