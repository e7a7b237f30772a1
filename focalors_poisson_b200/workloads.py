"""Synthetic composite-geometry workloads (geometry descriptions + seeded right-hand sides).

These are the shapes the solver is measured and checked on:

* ``cross``      centre + 4 arms (W, E, S, N) of n x n cells each, optional Neumann arm tips;
* ``lt_shape``   L (3 subdomains) or T (4 subdomains) shapes with uneven side lengths;
* ``tree9``      centre + 4 arms + 4 corner blocks, each corner attached to one arm (a tree: the
                 reference's geometry tree cannot hold cycles, base/domain/geometry_tree.hpp:136-160),
                 arms W and E periodic in y.

Boundary codes follow the reference's PDEBoundaryType (base/location_boundary.h:62-69) and faces its
LocationType order (XNegative, XPositive, YNegative, YPositive).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

DIRICHLET, NEUMANN, PERIODIC, ADJACENTED = 0, 1, 2, 3
XNEG, XPOS, YNEG, YPOS = 0, 1, 2, 3


def opposite(loc: int) -> int:
    return (XPOS, XNEG, YPOS, YNEG)[loc]


@dataclass
class Geometry:
    """A tree of uniform rectangles. bc[i][face] is the boundary type of every outer face; faces named by
    a connection are overwritten with ADJACENTED (Variable2D::set_geometry, variable2d.cpp:25-45)."""

    nx: list
    ny: list
    hx: list
    hy: list
    bc: list
    connections: list  # (a, loc, b): b lies at side `loc` of a
    offsets: list = field(default_factory=list)
    names: list = field(default_factory=list)

    def __post_init__(self):
        self.bc = [list(b) for b in self.bc]
        for a, loc, b in self.connections:
            self.bc[a][loc] = ADJACENTED
            self.bc[b][opposite(loc)] = ADJACENTED
        if not self.offsets:
            self.offsets = [(0.0, 0.0)] * len(self.nx)
        if not self.names:
            self.names = [f"D{i}" for i in range(len(self.nx))]

    @property
    def n_domains(self) -> int:
        return len(self.nx)

    def cells(self) -> int:
        return int(sum(a * b for a, b in zip(self.nx, self.ny)))

    def centres(self, i: int):
        x = self.offsets[i][0] + (np.arange(self.nx[i]) + 0.5) * self.hx[i]
        y = self.offsets[i][1] + (np.arange(self.ny[i]) + 0.5) * self.hy[i]
        return np.meshgrid(x, y, indexing="ij")


def cross(n: int, h: float | None = None, neumann_tips: bool = False, length: float = 1.0) -> Geometry:
    """Centre C (index 0) with arms W, E, S, N (1..4) of n x n cells, h = length / n. C sits at [1,2]^2 in
    units of `length` (Geometry2D::axis placement, geometry2d.cpp:186-215)."""
    h = length / n if h is None else h
    L = n * h
    bc = [[DIRICHLET] * 4 for _ in range(5)]
    if neumann_tips:
        bc[1][XNEG] = NEUMANN
        bc[2][XPOS] = NEUMANN
        bc[3][YNEG] = NEUMANN
        bc[4][YPOS] = NEUMANN
    conns = [(0, XNEG, 1), (0, XPOS, 2), (0, YNEG, 3), (0, YPOS, 4)]
    offs = [(L, L), (0.0, L), (2 * L, L), (L, 0.0), (L, 2 * L)]
    return Geometry([n] * 5, [n] * 5, [h] * 5, [h] * 5, bc, conns, offs, ["C", "W", "E", "S", "N"])


def cross_config1_rhs(g: Geometry) -> list:
    """sin(pi x) sin(pi y) at cell centres (Variable2D::set_value, variable2d.cpp:467-511). The seeded
    interior noise of the 128^2 cross case is added by the caller."""
    out = []
    for i in range(g.n_domains):
        X, Y = g.centres(i)
        out.append(np.sin(math.pi * X) * np.sin(math.pi * Y))
    return out


def gaussian_rhs(g: Geometry, seed: int, zero_mean: bool = True) -> list:
    """Seeded N(0,1) per cell, minus the global mean over all subdomains when zero_mean."""
    rng = np.random.default_rng(seed)
    f = [rng.standard_normal((a, b)) for a, b in zip(g.nx, g.ny)]
    if zero_mean:
        mean = sum(x.sum() for x in f) / g.cells()
        f = [x - mean for x in f]
    return f


SIDES = list(range(64, 1025, 32))


def lt_shape(seed: int, sides=None, h: float | None = None) -> Geometry:
    """One L- (3 subdomains) or T-shape (4 subdomains); free side lengths drawn uniformly from `sides`
    ({64, 96, ..., 1024} by default); all outer faces Dirichlet. A is index 0 (the tree root)."""
    sides = SIDES if sides is None else sides
    rng = np.random.default_rng(seed)
    kind = "L" if rng.integers(2) == 0 else "T"
    pick = lambda: int(sides[rng.integers(len(sides))])  # noqa: E731
    a, b = pick(), pick()
    hh = 1.0 / max(a, b) if h is None else h
    if kind == "L":
        nx = [a, pick(), a]
        ny = [b, b, pick()]
        conns = [(0, XPOS, 1), (0, YPOS, 2)]
    else:
        nx = [a, pick(), pick(), a]
        ny = [b, b, b, pick()]
        conns = [(0, XNEG, 1), (0, XPOS, 2), (0, YNEG, 3)]
    nd = len(nx)
    return Geometry(nx, ny, [hh] * nd, [hh] * nd, [[DIRICHLET] * 4 for _ in range(nd)], conns)


def tree9(n: int, h: float | None = None) -> Geometry:
    """Centre C(0), arms W(1) E(2) S(3) N(4), corners NW(5) NE(6) attached to N in x, SW(7) SE(8) attached to
    S in x. Arms W and E are periodic in y; arm tips Neumann; every other outer face Dirichlet."""
    h = 1.0 / n if h is None else h
    bc = [[DIRICHLET] * 4 for _ in range(9)]
    bc[1][YNEG] = bc[1][YPOS] = PERIODIC
    bc[2][YNEG] = bc[2][YPOS] = PERIODIC
    bc[1][XNEG] = NEUMANN
    bc[2][XPOS] = NEUMANN
    bc[3][YNEG] = NEUMANN
    bc[4][YPOS] = NEUMANN
    conns = [(0, XNEG, 1), (0, XPOS, 2), (0, YNEG, 3), (0, YPOS, 4), (4, XNEG, 5), (4, XPOS, 6), (3, XNEG, 7),
             (3, XPOS, 8)]
    L = n * h
    offs = [(L, L), (0, L), (2 * L, L), (L, 0), (L, 2 * L), (0, 2 * L), (2 * L, 2 * L), (0, 0), (2 * L, 0)]
    return Geometry([n] * 9, [n] * 9, [h] * 9, [h] * 9, bc, conns, offs,
                    ["C", "W", "E", "S", "N", "NW", "NE", "SW", "SE"])


def tree9_large(n: int = 4096) -> Geometry:
    """The large composite workload: the 9-subdomain tree of tree9 (n x n cells each, h = 1/n), arms W and E
    periodic in y, Neumann on the x faces of the W / E arm tips and of the four corners' outer x faces,
    Dirichlet on every other outer face. (No y-face Neumann: a quarter-wave y-transform of 4096 rows does
    not fit one CTA's shared memory in FP64.)"""
    g = tree9(n)
    g.bc[3][YNEG] = DIRICHLET
    g.bc[4][YPOS] = DIRICHLET
    for c, face in ((5, XNEG), (6, XPOS), (7, XNEG), (8, XPOS)):
        g.bc[c][face] = NEUMANN
    return g


def gaussian_bumps_rhs(g: Geometry, seed: int, n_bumps: int = 32, device=None) -> list:
    """Sum of seeded Gaussian bumps over the geometry's bounding box: centres uniform, widths U(0.01,0.05)
    times the box size, amplitudes N(0,1)."""
    rng = np.random.default_rng(seed)
    x0 = min(o[0] for o in g.offsets)
    y0 = min(o[1] for o in g.offsets)
    x1 = max(o[0] + a * h for o, a, h in zip(g.offsets, g.nx, g.hx))
    y1 = max(o[1] + b * h for o, b, h in zip(g.offsets, g.ny, g.hy))
    size = max(x1 - x0, y1 - y0)
    cx = rng.uniform(x0, x1, n_bumps)
    cy = rng.uniform(y0, y1, n_bumps)
    w = rng.uniform(0.01, 0.05, n_bumps) * size
    amp = rng.standard_normal(n_bumps)
    if device is not None:  # the same sum evaluated on a torch device (large fields)
        import torch

        out = []
        for i in range(g.n_domains):
            xs = torch.tensor(g.offsets[i][0] + (np.arange(g.nx[i]) + 0.5) * g.hx[i], device=device)
            ys = torch.tensor(g.offsets[i][1] + (np.arange(g.ny[i]) + 0.5) * g.hy[i], device=device)
            f = torch.zeros(g.nx[i], g.ny[i], dtype=torch.float64, device=device)
            for k in range(n_bumps):
                ex = torch.exp(-((xs - cx[k]) ** 2) / (2.0 * w[k] ** 2))
                ey = torch.exp(-((ys - cy[k]) ** 2) / (2.0 * w[k] ** 2))
                f += amp[k] * torch.outer(ex, ey)
            out.append(f)
        return out
    out = []
    for i in range(g.n_domains):
        X, Y = g.centres(i)
        f = np.zeros_like(X)
        for k in range(n_bumps):
            f += amp[k] * np.exp(-((X - cx[k]) ** 2 + (Y - cy[k]) ** 2) / (2.0 * w[k] ** 2))
        out.append(f)
    return out


def adjoint_case(n: int = 512, seed: int = 2024, probes: int = 64):
    """Differentiable-solve workload: cross 5 x n^2, h = 1/n, homogeneous Dirichlet outer faces; RHS
    f ~ N(0,1) (seed), per-cell source scale s ~ U(0.5, 1.5) (seed+1), target u_t ~ N(0,1) (seed+2), loss
    0.5 |u - u_t|^2 with u the solution for s*f; `probes` random cells (domain, i, j) (seed+3) for the
    finite-difference check."""
    g = cross(n)
    f = gaussian_rhs(g, seed, zero_mean=False)
    rng = np.random.default_rng(seed + 1)
    s = [rng.uniform(0.5, 1.5, (a, b)) for a, b in zip(g.nx, g.ny)]
    rng = np.random.default_rng(seed + 2)
    ut = [rng.standard_normal((a, b)) for a, b in zip(g.nx, g.ny)]
    rng = np.random.default_rng(seed + 3)
    dom = rng.integers(0, g.n_domains, probes)
    pts = [(int(d), int(rng.integers(0, g.nx[d])), int(rng.integers(0, g.ny[d]))) for d in dom]
    return g, f, s, ut, pts


SIDES = tuple(range(64, 1025, 32))  # {64, 96, ..., 1024}: 31 side lengths


def lt_problem(seed: int, sides=SIDES) -> Geometry:
    """One problem of the batched-uneven workload: an L (3 subdomains) or T (4 subdomains) shape, free side
    lengths drawn uniformly from `sides` with numpy default_rng(seed), homogeneous Dirichlet outer faces,
    one grid step h = 1/max(side) for every subdomain. Centre C (index 0) is the tree root.

      L: C (a x b); X at C's x+ face (c x b); Y at C's y+ face (a x d)
      T: C (a x b); W at C's x- face (c x b); E at C's x+ face (e x b); N at C's y+ face (a x d)
    """
    rng = np.random.default_rng(seed)
    shape = "L" if rng.integers(0, 2) == 0 else "T"
    draw = lambda: int(sides[rng.integers(0, len(sides))])  # noqa: E731
    a, b, c, d = draw(), draw(), draw(), draw()
    if shape == "L":
        nx, ny = [a, c, a], [b, b, d]
        conns = [(0, XPOS, 1), (0, YPOS, 2)]
        names = ["C", "X", "Y"]
    else:
        e = draw()
        nx, ny = [a, c, e, a], [b, b, b, d]
        conns = [(0, XNEG, 1), (0, XPOS, 2), (0, YPOS, 3)]
        names = ["C", "W", "E", "N"]
    h = 1.0 / max(nx + ny)
    nd = len(nx)
    return Geometry(nx, ny, [h] * nd, [h] * nd, [[DIRICHLET] * 4 for _ in range(nd)], conns, [(0.0, 0.0)] * nd,
                    names)


def batched_uneven(count: int = 512, seed: int = 2024, rhs: bool = True):
    """The batched-uneven workload: `count` independent L/T problems (problem p uses seed + p) and their
    seeded N(0,1) right-hand sides (seed + p + 1000003; None with rhs=False)."""
    geos = [lt_problem(seed + p) for p in range(count)]
    if not rhs:
        return geos, None
    return geos, [gaussian_rhs(g, seed + p + 1000003, zero_mean=False) for p, g in enumerate(geos)]

