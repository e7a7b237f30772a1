"""Subtree decomposition of the composite solve over GPUs: one process per GPU, torch.distributed (NCCL) for
the exchanges.

The reference decomposes its composite solve over MPI ranks (pe/concat/concat_solver2d_slab_x.cpp:381-402,
gmres_solver2d_slab_x.cpp:170-211). Here the tree of subdomains is cut at the root: rank 0 solves the root
domain, and every subtree hanging off a face of the root is a part of its own, given to one rank (largest
subtrees first, each to the least loaded rank by cells). ConcatPoissonSolver2D::solve
(pe/concat/concat_solver2d.cpp:101-157) then splits into

  1. every subtree part: boundary assembly, hx^2 scaling and the upward pass including its own root
     (fp_composite_part_upward), whose solved copy along the shared face is sent to rank 0;
  2. rank 0: its own assembly, the received vectors subtracted along the faces, the root's GMRES with the
     children's Schur matrices (fp_composite_root_solve), the root's solution along each face sent back;
  3. every subtree part: the received vector subtracted along its face, then its root's solve and the
     downward pass (fp_composite_part_downward).

So a solve exchanges one interface vector each way per subtree, and the root's Krylov iterations need no
exchange: the Schur matrices are computed once by the subtree parts (fp_composite_part_schur) and sent to
rank 0 at set-up. The answer is the undivided Schur GMRES solve's (capi.Composite(..., spectral=False)).

Every rank runs the same plan (computed from the geometry alone) and issues its sends and receives in the
same order. With one rank, every part lives on rank 0 and the exchange is a local hand-over.
"""
from __future__ import annotations

from dataclasses import dataclass, field as dc_field
from types import SimpleNamespace

ADJ = 3  # PDEBoundaryType::Adjacented


def tree_of(nd: int, connections, root: int = -1):
    """The composite solver's tree (the C ABI's build_tree, base/domain/geometry_tree.hpp:22-200): the root is
    the tree centre found by leaf stripping, a tie going to the lower domain index; children in face order.
    Returns (root, children: d -> [(face of d, child)], parent: child -> (face of child, parent))."""
    adj = [[-1] * 4 for _ in range(nd)]
    for a, f, b in connections:
        adj[a][f] = b
        adj[b][f ^ 1] = a
    if root < 0:
        if nd == 1:
            root = 0
        else:
            deg = [sum(1 for v in adj[d] if v >= 0) for d in range(nd)]
            leaves = [d for d in range(nd) if deg[d] <= 1]
            remaining = nd
            while remaining > 2 and leaves:
                remaining -= len(leaves)
                nxt = []
                for lf in leaves:
                    for v in adj[lf]:
                        if v >= 0:
                            deg[v] -= 1
                            if deg[v] == 1:
                                nxt.append(v)
                leaves = nxt
            root = min(leaves) if leaves else 0
    children = {d: [] for d in range(nd)}
    parent = {}
    stack, par = [root], {root: -1}
    while stack:
        u = stack.pop()
        for f in range(4):
            v = adj[u][f]
            if v < 0 or v == par[u]:
                continue
            par[v] = u
            children[u].append((f, v))
            parent[v] = (f ^ 1, u)
            stack.append(v)
    return root, children, parent


@dataclass
class Part:
    """A subtree under face `face` of the root: `domains` (global indices, the subtree root first), its local
    geometry, the rank that solves it."""

    face: int
    child: int
    domains: list
    geo: SimpleNamespace
    rank: int = 0
    cells: int = 0


@dataclass
class Plan:
    root: int
    root_geo: SimpleNamespace
    parts: list = dc_field(default_factory=list)  # in the root's face order

    def owned(self, rank):
        return [p for p in self.parts if p.rank == rank]


def make_plan(geo, world: int, root: int = -1) -> Plan:
    """The decomposition of `geo` (nx, ny, hx, hy, bc, connections per domain, as capi.Composite takes) over
    `world` ranks: the root domain on rank 0, each subtree of the root to one rank (ranks 1.. when there are
    several ranks, rank 0 otherwise), largest subtrees first to the least loaded rank."""
    nd = len(geo.nx)
    r, children, _ = tree_of(nd, geo.connections, root)
    conns = list(geo.connections)

    def sub(domains, conns_local, bc_local, local_root):
        return SimpleNamespace(nx=[geo.nx[d] for d in domains], ny=[geo.ny[d] for d in domains],
                               hx=[geo.hx[d] for d in domains], hy=[geo.hy[d] for d in domains], bc=bc_local,
                               connections=conns_local, root=local_root)

    root_bc = [list(geo.bc[r])]
    root_geo = sub([r], [], root_bc, 0)
    plan = Plan(r, root_geo)
    for face, c in children[r]:
        doms, stack = [], [c]
        while stack:
            u = stack.pop()
            doms.append(u)
            stack.extend(v for _, v in reversed(children[u]))
        index = {d: i for i, d in enumerate(doms)}
        local = [(index[a], f, index[b]) for a, f, b in conns if a in index and b in index]
        bc = [list(geo.bc[d]) for d in doms]
        bc[0][face ^ 1] = ADJ  # the face toward the root domain
        cells = sum(int(geo.nx[d]) * int(geo.ny[d]) for d in doms)
        plan.parts.append(Part(face, c, doms, sub(doms, local, bc, 0), cells=cells))
    if world > 1:
        load = [0] * world
        load[0] = int(geo.nx[r]) * int(geo.ny[r])
        for p in sorted(plan.parts, key=lambda q: -q.cells):
            rk = min(range(1, world), key=lambda q: (load[q], q))
            p.rank = rk
            load[rk] += p.cells
    return plan


class Exchange:
    """Point-to-point transfers between ranks: torch.distributed send / recv (NCCL for CUDA tensors, gloo for
    host tensors), and a local hand-over when both ends are this rank."""

    def __init__(self, rank: int, dist=None):
        self.rank, self.dist, self.box = rank, dist, {}

    def send(self, tensor, dst: int, tag):
        if dst == self.rank:
            self.box[tag] = tensor.clone()
        else:
            self.dist.send(tensor, dst)

    def recv(self, tensor, src: int, tag):
        if src == self.rank:
            tensor.copy_(self.box.pop(tag))
        else:
            self.dist.recv(tensor, src)


class SubtreeSolver:
    """The composite solve of `geo` split over ranks as `make_plan` says. `make_part(geo, ext_faces)` builds a
    part solver with the methods of capi.CompositePart (schur, set_external_schur, upward, downward,
    root_solve); `zeros(shape)` allocates the exchange buffers on the parts' device. Each rank holds the fields
    of the domains it owns: the root domain on rank 0, the domains of its parts elsewhere."""

    def __init__(self, geo, rank: int, world: int, make_part, zeros, dist=None, root: int = -1):
        self.plan = make_plan(geo, world, root)
        self.rank, self.world, self.zeros = rank, world, zeros
        self.ex = Exchange(rank, dist)
        p = self.plan
        self.edge_len = [int(geo.ny[p.root]) if q.face < 2 else int(geo.nx[p.root]) for q in p.parts]
        self.root_part = make_part(p.root_geo, [q.face for q in p.parts]) if rank == 0 else None
        self.mine = {k: make_part(q.geo, []) for k, q in enumerate(p.parts) if q.rank == rank}
        # set-up: every subtree part's Schur matrix toward the root domain goes to rank 0
        for k, q in enumerate(p.parts):
            n = self.edge_len[k]
            if k in self.mine:
                S = zeros((n, n))
                self.mine[k].schur(q.face ^ 1, S)
                self.ex.send(S, 0, ("S", k))
            if rank == 0:
                S = zeros((n, n))
                self.ex.recv(S, q.rank, ("S", k))
                self.root_part.set_external_schur(k, S)

    def owned_domains(self):
        """Global indices of the domains whose fields this rank passes to solve()."""
        out = [self.plan.root] if self.rank == 0 else []
        for k in sorted(self.mine):
            out.extend(self.plan.parts[k].domains)
        return out

    def solve(self, fields: dict, ghosts: dict | None = None):
        """fields: global domain index -> field tensor (in place) for owned_domains(); ghosts: the same keys ->
        four ghost tensors or None. Returns the root GMRES's info on rank 0, None elsewhere."""
        p = self.plan
        g = ghosts or {}
        edges = {}
        for k in sorted(self.mine):
            q = p.parts[k]
            e = self.zeros((self.edge_len[k],))
            self.mine[k].upward([fields[d] for d in q.domains], self._ghosts(q.domains, g), q.face ^ 1, e)
            self.ex.send(e, 0, ("up", k))
            edges[k] = e
        info = None
        if self.rank == 0:
            child = [self.zeros((n,)) for n in self.edge_len]
            out = [self.zeros((n,)) for n in self.edge_len]
            for k, q in enumerate(p.parts):
                self.ex.recv(child[k], q.rank, ("up", k))
            info = self.root_part.root_solve([fields[p.root]], self._ghosts([p.root], g), child, out)
            for k, q in enumerate(p.parts):
                self.ex.send(out[k], q.rank, ("down", k))
        for k in sorted(self.mine):
            q = p.parts[k]
            e = self.zeros((self.edge_len[k],))
            self.ex.recv(e, 0, ("down", k))
            self.mine[k].downward([fields[d] for d in q.domains], q.face ^ 1, e)
        return info

    @staticmethod
    def _ghosts(domains, g):
        if not any(g.get(d) is not None for d in domains):
            return None
        return [g.get(d) for d in domains]
