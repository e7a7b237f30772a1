"""Generate the golden fixtures in tests/golden/ from the reference's own sources built for CPU.

Run here (where the reference checkout and oracle/_ref/libfpref.so exist):

    make -C oracle && python tests/golden/make_golden.py

Every output array is produced by the reference's C++ (oracle/ref_harness.cpp over the unmodified
reference sources). Inputs follow the reference's own validation drivers where one exists
(case/validation/2d/poisson_solver_reference.cpp, concat_solver_reference.cpp, gmres_reference.cpp,
shur_mat_reference.cpp) and the benchmark workloads' shapes otherwise (seeded, synthetic), at sizes small
enough to commit. Files are .npz (little-endian float64 / int32 arrays).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refbind as R  # noqa: E402
from focalors_poisson_b200 import workloads as W  # noqa: E402

D, N, P, ADJ = 0, 1, 2, 3


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB")


def ref_order_combos():
    """The 25 boundary combinations of poisson_solver_reference.cpp:45-92, in its order."""
    combos = []
    for tn in range(4, -1, -1):
        for mask in range(16):
            if bin(mask).count("1") == tn:
                combos.append(tuple(N if (mask >> i) & 1 else D for i in range(4)))
    combos.append((P, P, P, P))
    for mask in range(4):
        combos.append((P, P, N if mask & 1 else D, N if mask & 2 else D))
    for mask in range(4):
        combos.append((N if mask & 1 else D, N if mask & 2 else D, P, P))
    return combos


def transforms():
    rng = np.random.default_rng(101)
    out = {}
    pairs = {"DD": (D, D), "NN": (N, N), "ND": (N, D), "DN": (D, N), "PP": (P, P)}
    for ny in [2, 3, 4, 5, 7, 8, 16, 31, 64, 100, 129, 257]:
        f = rng.standard_normal((3, ny))
        for k, (bn, bp) in pairs.items():
            if k == "PP" and ny % 2:
                continue
            out[f"in_{k}_{ny}"] = f
            out[f"fwd_{k}_{ny}"] = R.transform(bn, bp, f, False)
            out[f"inv_{k}_{ny}"] = R.transform(bn, bp, f, True)
    save("transforms.npz", **out)


def poisson():
    combos = ref_order_combos()
    out = {"combos": np.asarray(combos, dtype=np.int32)}
    # The reference driver itself: nx=3, ny=4, `int hx = 1.0; int hy = 2.0;` (:11-14), f = i*ny + j + 1.
    f = (np.arange(12, dtype=np.float64).reshape(3, 4) + 1.0)
    for c, bc in enumerate(combos):
        out[f"fixture_{c}"] = R.poisson2d_solve(f, 1.0, 2.0, bc)[0]
    rng = np.random.default_rng(202)
    for tag, (nx, ny, hx, hy) in {"a": (17, 24, 0.05, 0.04), "b": (32, 30, 1 / 32, 1 / 30)}.items():
        f = rng.standard_normal((nx, ny))
        out[f"rand_{tag}_in"] = f
        out[f"rand_{tag}_shape"] = np.array([nx, ny, 0, 0], dtype=np.float64)
        out[f"rand_{tag}_shape"][2:] = [hx, hy]
        for c, bc in enumerate(combos):
            if bc[2] == P and ny % 2:
                continue
            out[f"rand_{tag}_{c}"] = R.poisson2d_solve(f, hx, hy, bc)[0]
    save("poisson.npz", **out)


def poisson3d():
    """PoissonSolver3D (pe/poisson/poisson_solver3d.cpp:3-123) of the reference's own sources on seeded random
    fields: every x pair of {DD, NN, PP, DN} with every y and z pair of {DD, NN, DN, ND, PP}, 6 x 6 x 4 cells
    (nx, ny, nz), unequal spacings, and two cases of 64 cells along x (the partition chase)."""
    pairs = [(D, D), (N, N), (D, N), (N, D), (P, P)]
    rng = np.random.default_rng(303)
    out, combos = {}, []
    f = rng.standard_normal((6, 6, 4))
    out["small_in"] = f
    for bx in [(D, D), (N, N), (P, P), (D, N)]:
        for by in pairs:
            for bz in pairs:
                bc = bx + by + bz
                out[f"small_{len(combos)}"] = R.poisson3d_solve(f, 0.3, 0.2, 0.25, bc)[0]
                combos.append(bc)
    out["combos"] = np.asarray(combos, dtype=np.int32)
    for tag, (shape, h, bc) in {"a": ((64, 12, 10), (1 / 64, 1 / 12, 1 / 10), (D, N, P, P, D, D)),
                                 "b": ((64, 10, 8), (0.02, 0.03, 0.05), (N, N, N, N, N, N))}.items():
        g = rng.standard_normal(shape)
        out[f"{tag}_in"] = g
        out[f"{tag}_h"] = np.asarray(h)
        out[f"{tag}_bc"] = np.asarray(bc, dtype=np.int32)
        out[f"{tag}_out"] = R.poisson3d_solve(g, *h, bc)[0]
    save("poisson3d.npz", **out)


# 3D composite cases: domains (nx, ny, nz, lx, ly, lz), connections (a, face of a, b), outer boundary types per
# domain (6 faces x-, x+, y-, y+, z-, z+), whether ghost buffers are set.
CONCAT3D_CASES = {
    "pair": ([(16, 16, 16, 1.0, 1.0, 1.0), (12, 16, 16, 0.75, 1.0, 1.0)], [(0, 1, 1)],
             [[D] * 6, [D] * 6], False),
    "star": ([(12, 10, 8, 1.2, 1.0, 0.8), (8, 10, 8, 0.8, 1.0, 0.8), (12, 6, 8, 1.2, 0.6, 0.8),
              (12, 10, 5, 1.2, 1.0, 0.5), (12, 10, 4, 1.2, 1.0, 0.4)],
             [(0, 0, 1), (0, 3, 2), (0, 4, 3), (0, 5, 4)],
             [[D, N, D, D, D, D], [N, D, D, N, D, D], [D, D, D, N, N, D], [D, D, N, D, D, D], [N, D, D, D, D, N]], True),
    "chain": ([(6, 6, 6, 1.0, 1.0, 1.0)] * 4, [(0, 1, 1), (1, 1, 2), (2, 1, 3)],
              [[N, D, D, D, D, D], [D] * 6, [D] * 6, [D, N, N, N, N, N]], True),
    "periodic_y": ([(10, 8, 6, 1.0, 0.8, 0.6), (14, 8, 6, 1.4, 0.8, 0.6)], [(0, 1, 1)],
                   [[D, D, P, P, D, D], [D, N, P, P, D, D]], True),
    "x64": ([(64, 8, 8, 1.0, 0.125, 0.125), (32, 8, 8, 0.5, 0.125, 0.125)], [(0, 0, 1)],
            [[D, N, D, D, N, N], [D, D, D, D, D, D]], False),
}


def concat3d():
    """ConcatPoissonSolver3D (pe/concat/concat_solver3d.cpp) of the reference's own sources on seeded random
    right-hand sides and ghost buffers: two boxes, a star of four children on x-, y+, z- and z+ faces, a chain of
    four (a tree of depth 2), periodic y faces and a root of 64 cells along x (the partition chase); GMRES(20,
    1e-12, 100), and the same solve at tol 1e-15 ("tight")."""
    rng = np.random.default_rng(404)
    out = {}
    for name, (doms, conns, bcs, with_ghosts) in CONCAT3D_CASES.items():
        nx, ny, nz, lx, ly, lz = (list(v) for v in zip(*doms))
        rhs = [rng.standard_normal((a, b, c)) for a, b, c in zip(nx, ny, nz)]
        ghosts = None
        if with_ghosts:
            ghosts = [[rng.standard_normal(s) for s in ((b, c), (b, c), (a, c), (a, c), (a, b), (a, b))]
                      for a, b, c in zip(nx, ny, nz)]
        ref = R.Concat3DCase(nx, ny, nz, lx, ly, lz, conns, bcs, 20, 1e-12, 100)
        sol, _ = ref.solve(rhs, ghosts)
        tight, _ = R.Concat3DCase(nx, ny, nz, lx, ly, lz, conns, bcs, 20, 1e-15, 100).solve(rhs, ghosts)
        root, levels = ref.tree()
        out[f"{name}_dims"] = np.asarray(doms, dtype=np.float64)
        out[f"{name}_conns"] = np.asarray(conns, dtype=np.int32)
        out[f"{name}_bc"] = np.asarray(bcs, dtype=np.int32)
        out[f"{name}_root"] = np.asarray(root, dtype=np.int32)
        out[f"{name}_levels"] = levels
        for i in range(len(doms)):
            out[f"{name}_rhs_{i}"] = rhs[i]
            out[f"{name}_out_{i}"] = sol[i]
            out[f"{name}_tight_{i}"] = tight[i]
            for f in range(6):
                if ghosts is not None:
                    out[f"{name}_ghost_{i}_{f}"] = ghosts[i][f]
    save("concat3d.npz", **out)


def composite(name, g: W.Geometry, rhs, m, tol, max_iter, ghosts=None, extra=None):
    lx = [a * h for a, h in zip(g.nx, g.hx)]
    ly = [b * h for b, h in zip(g.ny, g.hy)]
    bc_outer = [[b if b != ADJ else D for b in row] for row in g.bc]
    case = R.ConcatCase(g.nx, g.ny, lx, ly, g.connections, bc_outer, m, tol, max_iter)
    root, levels = case.tree()
    outs, _ = case.solve(rhs, ghosts)
    # The same solve driven to tol 1e-15: the reference's own distance from the converged solution at
    # the configured tol bounds how closely any other Krylov iteration can agree with `outs`.
    tight = R.ConcatCase(g.nx, g.ny, lx, ly, g.connections, bc_outer, m, 1e-15, max_iter)
    touts, _ = tight.solve(rhs, ghosts)
    arrays = dict(
        nx=np.asarray(g.nx, np.int32), ny=np.asarray(g.ny, np.int32), hx=np.asarray(g.hx), hy=np.asarray(g.hy),
        bc=np.asarray(g.bc, np.int32), connections=np.asarray(g.connections, np.int32).reshape(-1, 3),
        gmres=np.array([m, tol, max_iter], dtype=np.float64), root=np.int32(root), levels=levels,
    )
    for i in range(g.n_domains):
        arrays[f"rhs_{i}"] = rhs[i]
        arrays[f"out_{i}"] = outs[i]
        arrays[f"tight_{i}"] = touts[i]
        if ghosts is not None:
            for f in range(4):
                if ghosts[i][f] is not None:
                    arrays[f"ghost_{i}_{f}"] = ghosts[i][f]
    if extra:
        arrays.update(extra)
    save(name, **arrays)


def fixture6():
    """case/validation/2d/concat_solver_reference.cpp:42-115 (T1 8x7 centre; T2 nx 7 at x-, T3 nx 8 at x+,
    T4 ny 8 at y-, T5 ny 7 at y+, T6 nx 8 at T3's x+; h = 1; all outer faces Dirichlet; f = i*ny + j + 1;
    default GMRES parameters m=20, tol=1e-8, maxIter=100)."""
    nx = [8, 7, 8, 8, 8, 8]
    ny = [7, 7, 7, 8, 7, 7]
    conns = [(0, W.XNEG, 1), (0, W.XPOS, 2), (0, W.YNEG, 3), (0, W.YPOS, 4), (2, W.XPOS, 5)]
    g = W.Geometry(nx, ny, [1.0] * 6, [1.0] * 6, [[D] * 4 for _ in range(6)], conns)
    rhs = [np.arange(a * b, dtype=np.float64).reshape(a, b) + 1.0 for a, b in zip(nx, ny)]
    composite("concat_fixture6.npz", g, rhs, 20, 1e-8, 100)
    composite("concat_fixture6_tight.npz", g, rhs, 20, 1e-12, 100)


def cross_config1():
    """Cross 5 x 128^2, h = 1/128, Dirichlet 0, sin(pi x) sin(pi y) plus add_random_number(+-1e-3) with
    seeds 1..5 in domain order C, W, E, S, N; GMRES(20, 1e-12, 100)."""
    g = W.cross(128)
    rhs = [R.add_random(f, -1e-3, 1e-3, i + 1) for i, f in enumerate(W.cross_config1_rhs(g))]
    composite("cross128_dirichlet.npz", g, rhs, 20, 1e-12, 100)


def cross_neumann():
    g = W.cross(48, neumann_tips=True)
    composite("cross48_neumann_tips.npz", g, W.gaussian_rhs(g, 7), 20, 1e-12, 100)


def cross_ghosts():
    """Non-zero Dirichlet and Neumann ghost buffers (boundary_assembly, concat_solver2d.cpp:159-223)."""
    g = W.cross(24, neumann_tips=True)
    rng = np.random.default_rng(303)
    ghosts = []
    for i in range(5):
        row = []
        for f in range(4):
            n = g.ny[i] if f < 2 else g.nx[i]
            row.append(None if g.bc[i][f] == ADJ else rng.standard_normal(n))
        ghosts.append(row)
    composite("cross24_ghosts.npz", g, W.gaussian_rhs(g, 8, zero_mean=False), 20, 1e-12, 100, ghosts=ghosts)


def cross64():
    """Cross 5 x 64^2 (a size the spectral path covers) with Neumann arm tips: quarter-wave (ND / DN)
    y-families on the y-arms, Neumann chase ends on the x-arms; once with zero ghosts, once with non-zero
    Dirichlet and Neumann ghost values."""
    g = W.cross(64, neumann_tips=True)
    composite("cross64_neumann_tips.npz", g, W.gaussian_rhs(g, 17), 20, 1e-12, 200)
    rng = np.random.default_rng(404)
    ghosts = [[None if g.bc[i][f] == ADJ else rng.standard_normal(g.ny[i] if f < 2 else g.nx[i]) for f in range(4)]
              for i in range(5)]
    composite("cross64_ghosts.npz", g, W.gaussian_rhs(g, 18, zero_mean=False), 20, 1e-12, 200, ghosts=ghosts)


def lt_shapes():
    for seed in range(4):
        g = W.lt_shape(seed, sides=[8, 12, 16, 20, 24, 32])
        composite(f"lt_shape_{seed}.npz", g, W.gaussian_rhs(g, 40 + seed, zero_mean=False), 20, 1e-12, 100)


def batch_lt():
    """Small problems of the batched-uneven workload (L and T shapes, sides 64 / 96 / 128), one of them
    with non-zero Dirichlet ghost values."""
    for k, seed in enumerate((11, 12, 13, 14)):
        g = W.lt_problem(seed, sides=(64, 96, 128))
        rhs = W.gaussian_rhs(g, 500 + seed, zero_mean=False)
        ghosts = None
        if k == 3:
            rng = np.random.default_rng(600)
            ghosts = [[None if g.bc[i][f] == ADJ or any(c[0] == i and c[1] == f or c[2] == i and c[1] == (f ^ 1)
                                                         for c in g.connections)
                       else rng.standard_normal(g.ny[i] if f < 2 else g.nx[i]) for f in range(4)]
                      for i in range(g.n_domains)]
        composite(f"batch_lt_{k}.npz", g, rhs, 20, 1e-12, 200, ghosts=ghosts)


def tree9():
    g = W.tree9(16)
    composite("tree9_periodic.npz", g, W.gaussian_bumps_rhs(g, 9), 20, 1e-12, 100)


def mocks():
    out = {}
    for loc in range(4):
        out[f"gmres_{loc}"] = R.gmres_mock(loc, 3, 5, 4, 2, 1e-3, 2)
    dims = [(6, 3, 4, 3), (6, 3, 4, 3), (3, 6, 3, 4), (3, 6, 3, 4)]  # shur_mat_reference.cpp:51-66
    for loc, (bnx, bny, nx, ny) in enumerate(dims):
        S, prod = R.schur_mock(loc, bnx, bny, nx, ny)
        out[f"schur_S_{loc}"] = S
        out[f"schur_prod_{loc}"] = prod
    save("mocks.npz", **out)


def dropin3d():
    """tests/cases/variable3d_case.cpp compiled against the reference's own headers and sources and run with
    "solve": per box the solution's sum, norm, first and last values (ConcatPoissonSolver3D, GMRES(20, 1e-13,
    100)) in the order the case prints them."""
    import subprocess
    import tempfile

    from oracle import refpath

    ref = refpath.reference_dir()
    src = os.path.join(ROOT, "tests", "cases", "variable3d_case.cpp")
    lib = os.path.join(ROOT, "oracle", "_ref")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "variable3d_ref")
        subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-I" + os.path.join(ROOT, "oracle", "shim"),
                        "-I" + ref, "-include", os.path.join(ref, "base", "pch.h"), src, "-o", exe, "-L" + lib,
                        "-lfpref", "-Wl,-rpath," + lib], check=True)
        out = subprocess.run([exe, "solve"], check=True, capture_output=True, text=True).stdout
    rows = [ln.split() for ln in out.splitlines() if ln.startswith("solution ")]
    save("dropin3d.npz", names=np.array([r[1] for r in rows]),
         values=np.array([[float(v) for v in r[2:]] for r in rows], dtype=np.float64))


if __name__ == "__main__":
    transforms()
    poisson()
    poisson3d()
    concat3d()
    fixture6()
    cross_config1()
    cross_neumann()
    cross_ghosts()
    lt_shapes()
    batch_lt()
    cross64()
    tree9()
    mocks()
    dropin3d()
