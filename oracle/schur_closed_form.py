"""Closed-form Schur matrices of leaf subdomains (numpy), for setting up the reference's solver at sizes
where its own construction is impractical on CPU.

TEST AND CPU-BASELINE INFRASTRUCTURE. The reference builds S for a child attached at face `loc` of its parent
with one full child solve per interface cell (pe/concat/schur_mat2d.cpp:5-106). For a leaf child the
response is separable:

* loc in {XNeg, XPos}: the interface runs along the child's transform axis y, so
  S = Psi diag(t) Phi, with Phi / Psi the child's forward / inverse y-transform matrices and t_k the
  diagonal entry of the k-th x-chase inverse at the interface row;
* loc in {YNeg, YPos}: the interface runs along x, and each x-chase matrix T_k = D_xx + (x_diag_k + 2) I
  is diagonalised by the x-transform of the child's x boundary pair, giving
  S = Psi_x diag(s) Phi_x with s_m = sum_k w_k / (lambda_x,m - 2 + x_diag_k + 2),
  w_k = Psi_y[y_if, k] Phi_y[k, y_if].

Everything is evaluated with oracle/fp_oracle.py's restatement of the reference's transforms and chase.
S[j, i] = response at interface cell j to a unit impulse at interface cell i (the reference's layout).
"""
from __future__ import annotations

import numpy as np

from . import fp_oracle as O


def _matrices(kind, n):
    eye = np.eye(n)
    phi = O.transform_forward(kind, eye).T  # f_hat = phi @ f
    psi = O.transform_inverse(kind, eye).T  # f = psi @ f_hat
    return phi, psi


def leaf_schur(loc: int, nx: int, ny: int, hx: float, hy: float, bc) -> np.ndarray:
    """Schur matrix of a leaf child (nx x ny cells, boundary types bc in face order, its face toward the
    parent Adjacented) attached at face `loc` of the parent."""
    bc = list(bc)
    kind_y = O.transform_kind(bc[2], bc[3])
    lam = O.cal_lambda(ny, bc[2], bc[3])
    xd = -2.0 + hx * hx / hy / hy * (lam - 2.0)
    phi, psi = _matrices(kind_y, ny)
    if loc in (O.XNEG, O.XPOS):
        x_if = nx - 1 if loc == O.XNEG else 0
        E = np.zeros((nx, ny))
        E[x_if, :] = 1.0
        t = O.chase(E, xd, False, bc[0], bc[1])[x_if, :]
        return psi @ (t[:, None] * phi)
    y_if = ny - 1 if loc == O.YNEG else 0
    w = psi[y_if, :] * phi[:, y_if]
    kind_x = O.transform_kind(bc[0], bc[1])
    mu = O.cal_lambda(nx, bc[0], bc[1]) - 2.0
    phx, psx = _matrices(kind_x, nx)
    s = (w[None, :] / (mu[:, None] + (xd[None, :] + 2.0))).sum(axis=1)
    return psx @ (s[:, None] * phx)


def root_schur_matrices(geo) -> list:
    """Per domain index: the Schur matrix the root's GMRES uses for that child (None for the root and for
    domains that are not children of the root). Every child of the root must be a leaf."""
    tree = O.build_tree(len(geo.nx), geo.connections)
    out = [None] * len(geo.nx)
    for loc, c in tree.children[tree.root]:
        if tree.children[c]:
            raise ValueError("closed form needs leaf children")
        bc = [O.D if b == O.ADJ else b for b in geo.bc[c]]
        bc[loc ^ 1] = O.ADJ
        out[c] = leaf_schur(loc, geo.nx[c], geo.ny[c], geo.hx[c], geo.hy[c], bc)
    return out
