"""The identity behind the adjoint solve, on the CPU oracle: the map f -> u of ConcatPoissonSolver2D::solve
(zero ghosts) is A^-1 H with A symmetric, so its transpose is H A^-1 = H solve(H^-1 .). Checked as a
dot-product test <solve(f), g> = <f, H solve(H^-1 g)> on geometries with unequal steps across interfaces."""
import numpy as np
import pytest

from adjoint_cases import CASES
from oracle import fp_oracle as O


def oracle_solver(geo):
    doms = [O.Domain(a, b, hx, hy, list(bc)) for a, b, hx, hy, bc in zip(geo.nx, geo.ny, geo.hx, geo.hy, geo.bc)]
    return O.ConcatPoissonSolver2D(doms, geo.connections, 20, 1e-14, 200)


@pytest.mark.parametrize("name", sorted(CASES))
def test_solve_map_is_self_adjoint_up_to_h2(name):
    geo = CASES[name]()
    solver = oracle_solver(geo)
    rng = np.random.default_rng(7)
    f = [rng.standard_normal((a, b)) for a, b in zip(geo.nx, geo.ny)]
    g = [rng.standard_normal((a, b)) for a, b in zip(geo.nx, geo.ny)]
    u = solver.solve([x.copy() for x in f])
    h2 = [hx * hx for hx in geo.hx]
    v = solver.solve([x / c for x, c in zip(g, h2)])
    v = [x * c for x, c in zip(v, h2)]
    lhs = sum(float((a * b).sum()) for a, b in zip(u, g))
    rhs = sum(float((a * b).sum()) for a, b in zip(f, v))
    scale = np.sqrt(sum(float((a * a).sum()) for a in u) * sum(float((b * b).sum()) for b in g))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)
    # the naive transpose (no H) is wrong as soon as the steps differ
    w = solver.solve([x.copy() for x in g])
    naive = sum(float((a * b).sum()) for a, b in zip(f, w))
    assert abs(lhs - naive) > 1e-6 * scale
