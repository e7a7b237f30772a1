"""Part solvers of the subtree decomposition (focalors_poisson_b200.decomp) built from the oracle, for CPU tests
of the decomposition's logic with gloo ranks (test infrastructure: numpy on torch CPU tensors, the same methods
as capi.CompositePart)."""
import numpy as np
import torch

from oracle import fp_oracle as O


def _edge(f, face):
    return {O.XNEG: f[0, :], O.XPOS: f[-1, :], O.YNEG: f[:, 0], O.YPOS: f[:, -1]}[face]


class OraclePart:
    def __init__(self, geo, ext_faces, m, tol, max_iter):
        doms = [O.Domain(int(nx), int(ny), float(hx), float(hy), list(bc))
                for nx, ny, hx, hy, bc in zip(geo.nx, geo.ny, geo.hx, geo.hy, geo.bc)]
        self.ext = list(ext_faces)
        self.m, self.tol, self.max_iter = m, tol, max_iter
        if self.ext:  # the root domain alone; its children's faces are Adjacented
            d = doms[0]
            bc = list(d.bc)
            for f in self.ext:
                bc[f] = O.ADJ
            self.dom = d
            self.bc = bc
            self.ps = O.PoissonSolver2D(d.nx, d.ny, d.hx, d.hy, bc)
            self.gmres = O.GMRESSolver2D(m, tol, max_iter, self.ps.solve)
            self.S = [None] * len(self.ext)
        else:
            self.c = O.ConcatPoissonSolver2D(doms, list(geo.connections), m, tol, max_iter, root=0)

    # subtree part -------------------------------------------------------------------------------------
    def schur(self, face, S):
        d = self.c.domains[0]
        S.copy_(torch.from_numpy(O.schur_matrix(face ^ 1, d.nx, d.ny, self.c.solvers[0])))

    def _assembled(self, fields, ghosts):
        f = [t.numpy().copy() for t in fields]
        gh = None if ghosts is None else [None if g is None else [None if x is None else x.numpy() for x in g]
                                          for g in ghosts]
        self.c.boundary_assembly(f, gh)
        for i, dom in enumerate(self.c.domains):
            f[i] *= dom.hx * dom.hx
        return f

    def upward(self, fields, ghosts, face, edge_out):
        f = self._assembled(fields, ghosts)
        T = self.c.tree
        temp = {}
        for lvl in reversed(T.levels[1:]):
            for d in lvl:
                temp[d] = f[d].copy()
                for loc, ch in T.children[d]:
                    O.bond_add(temp[d], loc, -1.0, temp[ch])
                    O.bond_add(f[d], loc, -1.0, temp[ch])
            for d in lvl:
                temp[d] = self.c.solvers[d](temp[d])
        t0 = f[0].copy()
        for loc, ch in T.children[0]:
            O.bond_add(t0, loc, -1.0, temp[ch])
            O.bond_add(f[0], loc, -1.0, temp[ch])
        t0 = self.c.solvers[0](t0)
        edge_out.copy_(torch.from_numpy(_edge(t0, face).copy()))
        for t, v in zip(fields, f):
            t.copy_(torch.from_numpy(v))

    def downward(self, fields, face, parent_edge):
        f = [t.numpy().copy() for t in fields]
        _edge(f[0], face)[...] -= parent_edge.numpy()
        T = self.c.tree
        f[0] = self.c.solvers[0](f[0])
        for lvl in T.levels[1:]:
            for d in lvl:
                ploc, par = T.parent[d]
                O.bond_add(f[d], ploc, -1.0, f[par])
            for d in lvl:
                f[d] = self.c.solvers[d](f[d])
        for t, v in zip(fields, f):
            t.copy_(torch.from_numpy(v))

    # root part ----------------------------------------------------------------------------------------
    def set_external_schur(self, k, S):
        self.S[k] = S.numpy().copy()
        self.gmres.S = [(f, s) for f, s in zip(self.ext, self.S) if s is not None]

    def root_solve(self, fields, ghosts, child_edges, edges_out):
        d = self.dom
        f = fields[0].numpy().copy()
        bt = self.bc
        g = None if ghosts is None or ghosts[0] is None else ghosts[0]

        def gv(face):
            v = None if g is None else g[face]
            return np.zeros(d.ny if face < 2 else d.nx) if v is None else v.numpy()

        for face, coef in ((O.XNEG, -1.0 / d.hx / d.hx), (O.XPOS, -1.0 / d.hx / d.hx),
                           (O.YNEG, -1.0 / d.hy / d.hy), (O.YPOS, -1.0 / d.hy / d.hy)):
            if bt[face] == O.D:
                O._edge_add(f, face, coef, gv(face))
        for face, coef in ((O.XNEG, 1.0 / d.hx), (O.XPOS, -1.0 / d.hx), (O.YNEG, 1.0 / d.hy), (O.YPOS, -1.0 / d.hy)):
            if bt[face] == O.N:
                O._edge_add(f, face, coef, gv(face))
        f *= d.hx * d.hx
        for face, e in zip(self.ext, child_edges):
            _edge(f, face)[...] -= e.numpy()
        f = self.gmres.solve(f)
        for face, e in zip(self.ext, edges_out):
            e.copy_(torch.from_numpy(_edge(f, face).copy()))
        fields[0].copy_(torch.from_numpy(f))
