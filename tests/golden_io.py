"""Loading helpers for the golden fixtures in tests/golden/ (written by tests/golden/make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def tight_outputs(name):
    """The reference's solution of the same case driven to GMRES tol 1e-15."""
    z = load(name)
    return [z[f"tight_{i}"] for i in range(len(z["nx"]))]


def composite_case(name):
    """Returns (geometry dict, rhs list, ghosts or None, outputs list, (m, tol, max_iter), root)."""
    z = load(name)
    nd = len(z["nx"])
    geo = dict(nx=[int(v) for v in z["nx"]], ny=[int(v) for v in z["ny"]], hx=[float(v) for v in z["hx"]],
               hy=[float(v) for v in z["hy"]], bc=[[int(b) for b in row] for row in z["bc"]],
               connections=[tuple(int(v) for v in c) for c in z["connections"]])
    rhs = [z[f"rhs_{i}"] for i in range(nd)]
    outs = [z[f"out_{i}"] for i in range(nd)]
    ghosts = None
    if any(k.startswith("ghost_") for k in z.files):
        ghosts = [[z[f"ghost_{i}_{f}"] if f"ghost_{i}_{f}" in z.files else None for f in range(4)] for i in range(nd)]
    m, tol, it = z["gmres"]
    return geo, rhs, ghosts, outs, (int(m), float(tol), int(it)), int(z["root"])


COMPOSITE_CASES = ["concat_fixture6.npz", "concat_fixture6_tight.npz", "cross128_dirichlet.npz",
                   "cross48_neumann_tips.npz", "cross24_ghosts.npz", "lt_shape_0.npz", "lt_shape_1.npz",
                   "lt_shape_2.npz", "lt_shape_3.npz", "tree9_periodic.npz", "cross64_neumann_tips.npz",
                   "cross64_ghosts.npz"]


def rel_l2(a_list, b_list):
    num = sum(float(((np.asarray(a) - np.asarray(b)) ** 2).sum()) for a, b in zip(a_list, b_list))
    den = sum(float((np.asarray(b) ** 2).sum()) for b in b_list)
    return (num / den) ** 0.5


CONCAT3D_CASES = ["pair", "star", "chain", "periodic_y", "x64"]


def concat3d_case(name):
    """Returns (domains [(nx, ny, nz, hx, hy, hz)], connections, bc per domain (6), rhs list, ghosts or None,
    outputs list (GMRES tol 1e-12), tight outputs (tol 1e-15), root, levels) of tests/golden/concat3d.npz."""
    z = load("concat3d.npz")
    dims = z[f"{name}_dims"]
    doms = [(int(d[0]), int(d[1]), int(d[2]), d[3] / d[0], d[4] / d[1], d[5] / d[2]) for d in dims]
    nd = len(doms)
    conns = [tuple(int(v) for v in c) for c in z[f"{name}_conns"]]
    bc = [[int(b) for b in row] for row in z[f"{name}_bc"]]
    rhs = [z[f"{name}_rhs_{i}"] for i in range(nd)]
    ghosts = None
    if f"{name}_ghost_0_0" in z.files:
        ghosts = [[z[f"{name}_ghost_{i}_{f}"] for f in range(6)] for i in range(nd)]
    outs = [z[f"{name}_out_{i}"] for i in range(nd)]
    tight = [z[f"{name}_tight_{i}"] for i in range(nd)]
    return doms, conns, bc, rhs, ghosts, outs, tight, int(z[f"{name}_root"]), z[f"{name}_levels"]
