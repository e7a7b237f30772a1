"""Subtree decomposition of the composite solve (focalors_poisson_b200.decomp) across ranks: run as three gloo
ranks on the CPU with the oracle's part solvers, the decomposed solve must equal the oracle's undivided
ConcatPoissonSolver2D solve; the plan must cover every domain once and follow the solver's tree rule."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from decomp_oracle import OraclePart
from focalors_poisson_b200 import decomp
from focalors_poisson_b200 import workloads as W
from oracle import fp_oracle as O

GMRES = (20, 1e-13, 100)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(name):
    if name == "tree9":
        g = W.tree9(12)
    else:
        g = W.cross(16, neumann_tips=True)
    rng = np.random.default_rng(7)
    rhs = [rng.standard_normal((nx, ny)) for nx, ny in zip(g.nx, g.ny)]
    ghosts = [[rng.standard_normal(ny), rng.standard_normal(ny), rng.standard_normal(nx), rng.standard_normal(nx)]
              for nx, ny in zip(g.nx, g.ny)]
    return g, rhs, ghosts


def _undivided(g, rhs, ghosts):
    doms = [O.Domain(nx, ny, hx, hy, list(bc)) for nx, ny, hx, hy, bc in zip(g.nx, g.ny, g.hx, g.hy, g.bc)]
    return O.ConcatPoissonSolver2D(doms, list(g.connections), *GMRES).solve(rhs, ghosts)


def _rank(rank, world, port, name, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, rhs, ghosts = _case(name)
        solver = decomp.SubtreeSolver(g, rank, world, lambda geo, ext: OraclePart(geo, ext, *GMRES),
                                      lambda shape: torch.zeros(shape, dtype=torch.float64), dist)
        mine = solver.owned_domains()
        fields = {d: torch.from_numpy(rhs[d].copy()) for d in mine}
        gh = {d: [torch.from_numpy(x.copy()) for x in ghosts[d]] for d in mine}
        solver.solve(fields, gh)
        out[rank] = {d: fields[d].numpy().copy() for d in mine}
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["cross", "tree9"])
def test_decomposed_solve_equals_undivided(name):
    world = 3
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), name, out), nprocs=world, join=True)
        res = dict(out)
    got = {}
    for r in range(world):
        for d, v in res[r].items():
            assert d not in got  # each domain solved by exactly one rank
            got[d] = v
    g, rhs, ghosts = _case(name)
    want = _undivided(g, rhs, ghosts)
    assert sorted(got) == list(range(len(g.nx)))
    num = sum(float(((got[d] - want[d]) ** 2).sum()) for d in got)
    den = sum(float((w ** 2).sum()) for w in want)
    assert (num / den) ** 0.5 <= 1e-13, name


def test_single_rank_plan_is_local():
    """One rank: every part on rank 0, hand-overs local; the oracle parts still give the undivided answer."""
    g, rhs, ghosts = _case("tree9")
    solver = decomp.SubtreeSolver(g, 0, 1, lambda geo, ext: OraclePart(geo, ext, *GMRES),
                                  lambda shape: torch.zeros(shape, dtype=torch.float64))
    fields = {d: torch.from_numpy(rhs[d].copy()) for d in solver.owned_domains()}
    solver.solve(fields, {d: [torch.from_numpy(x.copy()) for x in ghosts[d]] for d in fields})
    want = _undivided(g, rhs, ghosts)
    num = sum(float(((fields[d].numpy() - want[d]) ** 2).sum()) for d in fields)
    den = sum(float((w ** 2).sum()) for w in want)
    assert (num / den) ** 0.5 <= 1e-13


def test_plan_covers_domains_and_balances():
    g = W.tree9(64)
    tree = O.build_tree(len(g.nx), list(g.connections))
    for world in (1, 2, 3, 5, 8):
        p = decomp.make_plan(g, world)
        assert p.root == tree.root
        doms = [p.root] + [d for q in p.parts for d in q.domains]
        assert sorted(doms) == list(range(len(g.nx)))
        assert [q.face for q in p.parts] == sorted(q.face for q in p.parts)
        if world > 1:
            assert all(1 <= q.rank < world for q in p.parts)
        for q in p.parts:  # the subtree's face toward the root is Adjacented, its tree rooted at the child
            assert q.geo.bc[0][q.face ^ 1] == decomp.ADJ and q.domains[0] == q.child
