"""CPU restatement (numpy) of Focalors_Poisson's 2D composite FFT / domain-decomposition Poisson path.

TEST INFRASTRUCTURE -- the oracle. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
may import this module, and only as the checker. The product path never does.

Every function restates one reference routine (paths relative to the reference project):

* transforms        pe/poisson/poisson_fft2d.cpp:19-465  (PoissonFFT2D_{DD,NN,ND,DN,PP})
* cal_lambda        pe/poisson/poisson_solver2d_base.cpp:28-62
* x_diag / solve    pe/poisson/poisson_solver2d.cpp:37-90
* chasing           pe/poisson/chasing_method_base.cpp:24-279, pe/poisson/chasing_method2d.cpp:3-89
* bond_add          base/field/field2.cpp:212-302
* GMRES / Afun      pe/concat/gmres_solver2d.cpp:39-252
* Schur matrices    pe/concat/schur_mat2d.cpp:5-123
* composite solve   pe/concat/concat_solver2d.cpp:48-223
* tree / root       base/domain/geometry_tree.hpp:22-200 (root tie broken by lower domain index,
                    which equals the reference's lower-address rule for contiguously allocated domains)
* 3D rectangle      pe/poisson/poisson_solver3d.cpp:49-123, chasing_method3d.cpp:3-103
* 3D composite      pe/concat/concat_solver3d.cpp:5-247, gmres_solver3d.cpp:20-306,
                    schur_mat3d.cpp:5-285, base/field/field3.cpp:237-375

FFTW's r2c (the only third-party arithmetic; FFTW3, version unpinned by the reference) is restated by
numpy.fft.rfft, which has the same unnormalised forward definition. Parity of this module is pinned
against the reference's own sources built here (oracle/_ref, see oracle/Makefile) through the golden
fixtures in tests/golden/.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field as dc_field

import numpy as np

# PDEBoundaryType (base/location_boundary.h:62-69) and LocationType (:8-16) numbering.
D, N, P, ADJ, NULL = 0, 1, 2, 3, 4
XNEG, XPOS, YNEG, YPOS, ZNEG, ZPOS = 0, 1, 2, 3, 4, 5
PI = 3.14159265358979323846  # base/pch.h:13


def opposite(loc: int) -> int:
    return {XNEG: XPOS, XPOS: XNEG, YNEG: YPOS, YPOS: YNEG, ZNEG: ZPOS, ZPOS: ZNEG}[loc]


def is_dir_like(t: int) -> bool:
    """base/location_boundary.cpp:58."""
    return t in (D, ADJ)


def transform_kind(bn: int, bp: int) -> str:
    """PoissonSolver2DBase::create_fft, pe/poisson/poisson_solver2d_base.cpp:64-91."""
    if bn == P and bp == P:
        return "PP"
    if bn == N and bp == N:
        return "NN"
    if is_dir_like(bn) and is_dir_like(bp):
        return "DD"
    if is_dir_like(bn) and bp == N:
        return "DN"
    if bn == N and is_dir_like(bp):
        return "ND"
    raise ValueError(f"unsupported y boundary pair {bn},{bp}")


def _rfft(x):
    return np.fft.rfft(x, axis=-1)


def _alt(ny, even):
    j = np.arange(ny)
    return np.where(j % 2 == 0, even, -even).astype(np.float64)


def transform_forward(kind: str, f: np.ndarray) -> np.ndarray:
    """PoissonFFT2D_*::transform on an (nx, ny) row-major field; rows are independent."""
    f = np.asarray(f, dtype=np.float64)
    nx, ny = f.shape
    j = np.arange(ny, dtype=np.float64)
    if kind == "DD":  # poisson_fft2d.cpp:37-45
        ex = np.zeros((nx, 2 * ny + 2))
        ex[:, 1 : ny + 1] = f
        X = _rfft(ex)
        return -math.sqrt(2.0 / (1.0 + ny)) * X[:, 1 : ny + 1].imag
    if kind == "NN":  # poisson_fft2d.cpp:77-118
        sqr_2_n, sqr_n = math.sqrt(2.0 / ny), math.sqrt(1.0 / ny)
        cos_ipi = np.cos(PI * (j + 1.0) / ny / 2)
        sin_ipi = np.sin(PI * (j + 1.0) / ny / 2)
        ex = np.zeros((nx, 2 * ny))
        ex[:, 1 : ny + 1] = _alt(ny, -1.0) * f
        X = _rfft(ex)
        out = np.empty((nx, ny))
        Xi = X[:, 1:ny]
        out[:, : ny - 1] = sqr_2_n * (-1.0 * cos_ipi[: ny - 1] * Xi.imag - sin_ipi[: ny - 1] * Xi.real)
        acc = np.zeros(nx)
        for jj in range(ny):  # sequential sum, as the reference
            acc = acc + sqr_n * f[:, jj]
        out[:, ny - 1] = acc
        return out
    if kind == "ND":  # poisson_fft2d.cpp:153-190
        sqr = math.sqrt(4.0 / (2.0 * ny + 1.0))
        ang = 2.0 * ny * PI * (j + 1.0) / (2.0 * ny + 1.0)
        cb, sb = np.cos(ang), np.sin(ang)
        ex = np.zeros((nx, 2 * ny + 1))
        ex[:, 1 : ny + 1] = (_alt(ny, -1.0) * sqr) * f
        X = _rfft(ex)[:, 1 : ny + 1]
        return sb * X.real - cb * X.imag
    if kind == "DN":  # poisson_fft2d.cpp:223-251
        sqr = math.sqrt(4.0 / (2.0 * ny + 1.0))
        ex = np.zeros((nx, 2 * ny + 1))
        ex[:, 1 : ny + 1] = (_alt(ny, -1.0) * sqr) * f
        X = _rfft(ex)[:, 1 : ny + 1]
        return _alt(ny, 1.0) * X.imag
    if kind == "PP":  # poisson_fft2d.cpp:324-432
        h = ny // 2
        sqr = math.sqrt(2.0 / ny)
        cq = np.cos(PI * (2.0 * j + 1.0) / 4.0)
        sq = np.sin(PI * (2.0 * j + 1.0) / 4.0)
        exs = np.zeros((nx, ny))
        exs[:, 1:ny] = f[:, : ny - 1]
        S = _rfft(exs)
        ts = np.zeros((nx, ny))
        for jj in range(h):
            if jj < h - 1:
                ts[:, 2 * jj + 2] = -1.0 * S[:, h - jj - 1].imag
            ts[:, 2 * jj + 1] = -1.0 * S[:, h - jj - 1].imag
        exc = np.zeros((nx, ny))
        exc[:, 1:ny] = _alt(ny - 1, 1.0) * f[:, : ny - 1]
        C = _rfft(exc)
        tc = np.zeros((nx, ny))
        last = f[:, ny - 1]
        for jj in range(h):
            tc[:, 2 * jj] = last - C[:, jj].real
            tc[:, 2 * jj + 1] = last - C[:, jj + 1].real
        return sqr * (cq * ts + sq * tc)
    raise ValueError(kind)


def transform_inverse(kind: str, p_hat: np.ndarray) -> np.ndarray:
    """PoissonFFT2D_*::transform_transpose on an (nx, ny) field."""
    p_hat = np.asarray(p_hat, dtype=np.float64)
    nx, ny = p_hat.shape
    j = np.arange(ny, dtype=np.float64)
    if kind == "DD":  # poisson_fft2d.cpp:48-57, self-inverse
        return transform_forward("DD", p_hat)
    if kind == "NN":  # poisson_fft2d.cpp:120-133
        sqr_2_n, sqr_n = math.sqrt(2.0 / ny), math.sqrt(1.0 / ny)
        cos_ipi = np.cos(PI * (j + 1.0) / ny / 2)
        sin_ipi = np.sin(PI * (j + 1.0) / ny / 2)
        sg = _alt(ny, 1.0)
        ex = np.zeros((nx, 2 * ny))
        ex[:, 1 : ny + 1] = cos_ipi * p_hat
        Y = _rfft(ex)[:, 1 : ny + 1]
        p = sg * sqr_2_n * Y.imag
        ex[:, 1 : ny + 1] = sin_ipi * p_hat
        Z = _rfft(ex)[:, 1 : ny + 1]
        p = p + sg * sqr_2_n * Z.real
        return p + (sqr_2_n + sqr_n) * p_hat[:, ny - 1 : ny]
    if kind == "ND":  # poisson_fft2d.cpp:192-205
        sqr = math.sqrt(4.0 / (2.0 * ny + 1.0))
        ang = 2.0 * ny * PI * (j + 1.0) / (2.0 * ny + 1.0)
        cb, sb = np.cos(ang), np.sin(ang)
        ex = np.zeros((nx, 2 * ny + 1))
        ex[:, 1 : ny + 1] = sqr * sb * p_hat
        p = _rfft(ex)[:, 1 : ny + 1].real
        ex[:, 1 : ny + 1] = sqr * cb * p_hat
        p = p - _rfft(ex)[:, 1 : ny + 1].imag
        return _alt(ny, -1.0) * p
    if kind == "DN":  # poisson_fft2d.cpp:253-262
        return transform_forward("DN", p_hat)
    if kind == "PP":  # poisson_fft2d.cpp:434-465
        h = ny // 2
        sqr = math.sqrt(2.0 / ny)
        cq = np.cos(PI * (2.0 * j + 1.0) / 4.0)
        sq = np.sin(PI * (2.0 * j + 1.0) / 4.0)
        ce = np.zeros((nx, ny))
        co = np.zeros((nx, ny))
        se = np.zeros((nx, ny))
        so = np.zeros((nx, ny))
        for jj in range(h):
            ce[:, jj] = cq[2 * jj] * p_hat[:, 2 * jj]
            co[:, jj + 1] = cq[2 * jj + 1] * p_hat[:, 2 * jj + 1]
            se[:, h - jj] = sq[2 * jj] * p_hat[:, 2 * jj]
            so[:, h - jj - 1] = sq[2 * jj + 1] * p_hat[:, 2 * jj + 1]
        CE, CO, SE, SO = _rfft(ce), _rfft(co), _rfft(se), _rfft(so)
        fc = np.zeros((nx, ny))
        fs = np.zeros((nx, ny))
        sign = -1.0
        for jj in range(h):
            fc[:, jj] = sign * (CE[:, jj + 1].imag + CO[:, jj + 1].imag)
            fs[:, jj] = SE[:, jj + 1].real + SO[:, jj + 1].real
            sign = -sign
        for jj in range(h - 1):
            fc[:, h + jj] = -1.0 * fc[:, h - 2 - jj]
            fs[:, h + jj] = fs[:, h - 2 - jj]
        fs[:, ny - 1] = SE[:, 0].real + SO[:, 0].real
        return sqr * (fc + fs)
    raise ValueError(kind)


def cal_lambda(n: int, bn: int, bp: int) -> np.ndarray:
    """PoissonSolver2DBase::cal_lambda, pe/poisson/poisson_solver2d_base.cpp:28-62 (begin = 1)."""
    lam = np.empty(n)
    for i in range(1, n + 1):
        if bn == P and bp == P:
            lam[i - 1] = -2.0 * math.cos(2.0 * PI / n * math.floor(i / 2.0))
        elif bn == N and bp == N:
            lam[i - 1] = -2.0 * math.cos(PI / n * i)
        elif is_dir_like(bn) and is_dir_like(bp):
            lam[i - 1] = +2.0 * math.cos(PI / (n + 1) * i)
        elif (is_dir_like(bn) and bp == N) or (bn == N and is_dir_like(bp)):
            lam[i - 1] = -2.0 * math.cos(2.0 * PI * i / (2 * n + 1))
        else:
            raise ValueError("unsupported boundary pair")
    return lam


def chase(fh: np.ndarray, x_diag: np.ndarray, no_dirichlet: bool, bx_neg: int, bx_pos: int,
          sing_from: int | None = None) -> np.ndarray:
    """ChasingMethod2D::chasing on the transformed field fh (nx, ny): one tridiagonal system of length nx
    per wavenumber k (column), diagonal x_diag[k], unit off-diagonals.
    chasing_method2d.cpp:44-89; chasing_method_base.cpp:24-154 (standard / singular),
    :178-279 (periodic / periodic singular). Without a Dirichlet face the columns from sing_from on (the
    last one by default) take the singular recursions (ChasingMethod3D uses a range, see PoissonSolver3D)."""
    fh = np.asarray(fh, dtype=np.float64)
    n, K = fh.shape
    out = np.empty_like(fh)
    d = np.asarray(x_diag, dtype=np.float64)
    periodic = bx_neg == P and bx_pos == P
    sing = np.zeros(K, dtype=bool)
    if no_dirichlet:
        sing[(K - 1 if sing_from is None else sing_from):] = True  # has_last_vector: the last wavenumber(s)
    reg = ~sing

    def standard(f, dd, start_neu, end_neu):
        c = np.zeros((max(n - 1, 1), dd.shape[0]))
        y = np.zeros((n, dd.shape[0]))
        x = np.zeros((n, dd.shape[0]))
        c[0] = 1.0 / (dd + 1.0) if start_neu else 1.0 / dd
        for i in range(1, n - 1):
            c[i] = 1.0 / (dd - c[i - 1])
        y[0] = f[0] / (dd + 1.0) if start_neu else f[0] / dd
        for i in range(1, n - 1):
            y[i] = (f[i] - y[i - 1]) / (dd - c[i - 1])
        y[n - 1] = (f[n - 1] - y[n - 2]) / (dd + 1.0 - c[n - 2]) if end_neu else (f[n - 1] - y[n - 2]) / (dd - c[n - 2])
        x[n - 1] = y[n - 1]
        for i in range(n - 2, -1, -1):
            x[i] = y[i] - c[i] * x[i + 1]
        return x

    if periodic:
        dd = d[reg]
        e0 = np.zeros((n, dd.shape[0]))
        e0[0] = 1.0
        e1 = np.zeros((n, dd.shape[0]))
        e1[n - 1] = 1.0
        z1 = standard(e0, dd, False, False)
        z2 = standard(e1, dd, False, False)
        y = standard(fh[:, reg], dd, False, False)
        g2 = (y[n - 1] / (1.0 + z1[n - 1]) - y[0] / z1[0]) / (z2[n - 1] / (1.0 + z1[n - 1]) - (1.0 + z2[0]) / z1[0])
        g1 = y[0] / z1[0] - g2 * ((1.0 + z2[0]) / z1[0])
        out[:, reg] = y - g1 * z1 - g2 * z2
        for col in np.nonzero(sing)[0]:
            f = fh[:, col]
            x = np.zeros(n)
            x[0] = 0.0
            x1 = f[0] / n
            for i in range(1, n - 1):
                x1 = x1 - (n - 1 - i) * f[i] / n
            x[1] = x1
            for i in range(2, n):
                x[i] = f[i - 1] - x[i - 2] + 2.0 * x[i - 1]
            out[:, col] = x
    else:
        out[:, reg] = standard(fh[:, reg], d[reg], bx_neg == N, bx_pos == N)
        for col in np.nonzero(sing)[0]:
            f = fh[:, col]
            x = np.zeros(n)
            x[0] = 0.0
            x[1] = 0.0 + f[0]
            for i in range(2, n):
                x[i] = f[i - 1] - x[i - 2] + 2.0 * x[i - 1]
            out[:, col] = x
    return out


class PoissonSolver2D:
    """PoissonSolver2D (pe/poisson/poisson_solver2d.cpp:3-90). bc = (xneg, xpos, yneg, ypos)."""

    def __init__(self, nx, ny, hx, hy, bc):
        self.nx, self.ny, self.hx, self.hy = nx, ny, float(hx), float(hy)
        self.bc = tuple(bc)
        self.kind = transform_kind(bc[2], bc[3])
        lam = cal_lambda(ny, bc[2], bc[3])
        self.x_diag = -2.0 + self.hx * self.hx / self.hy / self.hy * (lam - 2.0)
        self.no_dirichlet = not any(is_dir_like(b) for b in bc)
        self.calls = 0

    def solve(self, f: np.ndarray) -> np.ndarray:
        fh = transform_forward(self.kind, f)
        uh = chase(fh, self.x_diag, self.no_dirichlet, self.bc[0], self.bc[1])
        self.calls += 1
        return transform_inverse(self.kind, uh)


def cal_lambda3(n: int, bn: int, bp: int) -> np.ndarray:
    """PoissonSolver3DBase::cal_lambda, pe/poisson/poisson_solver3d_base.cpp:41-74 (begin = 1): the 2D
    eigenvalues shifted by -2."""
    lam = np.empty(n)
    for i in range(1, n + 1):
        if bn == P and bp == P:
            lam[i - 1] = -2.0 - 2.0 * math.cos(2.0 * PI / n * math.floor(i / 2.0))
        elif bn == N and bp == N:
            lam[i - 1] = -2.0 - 2.0 * math.cos(PI / n * i)
        elif is_dir_like(bn) and is_dir_like(bp):
            lam[i - 1] = -2.0 + 2.0 * math.cos(PI / (n + 1) * i)
        elif (is_dir_like(bn) and bp == N) or (bn == N and is_dir_like(bp)):
            lam[i - 1] = -2.0 - 2.0 * math.cos(2.0 * PI * i / (2 * n + 1))
        else:
            raise ValueError("unsupported boundary pair")
    return lam


class PoissonSolver3D:
    """PoissonSolver3D (pe/poisson/poisson_solver3d.cpp:49-123) on a field3 f of shape (nx, ny, nz), z
    contiguous. bc = (x-, x+, y-, y+, z-, z+). z-transform (:98-99), y-transform after a transpose (:101-105),
    ChasingMethod3D along x over every (z-mode k, y-mode j) pair with x_diag[k][j] = -2 + (hx/hy)^2 lambda_y[j]
    + (hx/hz)^2 lambda_z[k] (:57-70, chasing_method3d.cpp:3-103), inverse transforms (:113-122). Without a
    Dirichlet face the singular systems are the last (k, j) pair, or with periodic x every j of the last k
    (chasing_method3d.cpp:55-90)."""

    def __init__(self, nx, ny, nz, hx, hy, hz, bc):
        self.shape = (nx, ny, nz)
        self.bc = tuple(bc)
        self.ky, self.kz = transform_kind(bc[2], bc[3]), transform_kind(bc[4], bc[5])
        ly, lz = cal_lambda3(ny, bc[2], bc[3]), cal_lambda3(nz, bc[4], bc[5])
        self.x_diag = -2.0 + float(hx) * float(hx) / float(hy) / float(hy) * ly[None, :] + \
            float(hx) * float(hx) / float(hz) / float(hz) * lz[:, None]  # [k][j]
        self.no_dirichlet = not any(is_dir_like(b) for b in bc)
        periodic_x = bc[0] == P and bc[1] == P
        self.sing_from = (nz - 1) * ny if periodic_x else nz * ny - 1

    def solve(self, f: np.ndarray) -> np.ndarray:
        nx, ny, nz = self.shape
        a = transform_forward(self.kz, np.asarray(f, dtype=np.float64).reshape(nx * ny, nz)).reshape(nx, ny, nz)
        b = transform_forward(self.ky, np.ascontiguousarray(a.transpose(0, 2, 1)).reshape(nx * nz, ny))
        u = chase(b.reshape(nx, nz * ny), self.x_diag.reshape(-1), self.no_dirichlet, self.bc[0], self.bc[1],
                  self.sing_from)
        c = transform_inverse(self.ky, u.reshape(nx * nz, ny)).reshape(nx, nz, ny)
        c = np.ascontiguousarray(c.transpose(0, 2, 1)).reshape(nx * ny, nz)
        return transform_inverse(self.kz, c).reshape(nx, ny, nz)


def bond_add(f: np.ndarray, loc: int, a: float, nb: np.ndarray) -> None:
    """field2::bond_add(LocationType, a, const field2&) -- field2.cpp:257-302 (in place)."""
    if loc == XNEG:
        f[0, :] += a * nb[nb.shape[0] - 1, :]
    elif loc == XPOS:
        f[f.shape[0] - 1, :] += a * nb[0, :]
    elif loc == YNEG:
        f[:, 0] += a * nb[:, nb.shape[1] - 1]
    elif loc == YPOS:
        f[:, f.shape[1] - 1] += a * nb[:, 0]
    else:
        raise ValueError(loc)


def schur_matrix(loc: int, bnx: int, bny: int, branch_solve) -> np.ndarray:
    """SchurMat2D_{xneg,xpos,ypos,yneg}::construct, schur_mat2d.cpp:5-106. Returns value (cn x cn)."""
    cn = bny if loc in (XNEG, XPOS) else bnx
    S = np.zeros((cn, cn))
    for i in range(cn):
        t = np.zeros((bnx, bny))
        if loc == XNEG:
            t[bnx - 1, i] = 1.0
        elif loc == XPOS:
            t[0, i] = 1.0
        elif loc == YPOS:
            t[i, 0] = 1.0
        else:
            t[i, bny - 1] = 1.0
        t = branch_solve(t)
        if loc == XNEG:
            S[:, i] = t[bnx - 1, :cn]
        elif loc == XPOS:
            S[:, i] = t[0, :cn]
        elif loc == YPOS:
            S[:, i] = t[:cn, 0]
        else:
            S[:, i] = t[:cn, bny - 1]
    return S


def schur_apply(loc: int, S: np.ndarray, root: np.ndarray) -> np.ndarray:
    """SchurMat2D_*::operator*, schur_mat2d.cpp:18-123: a zero root-sized field with one edge written."""
    R = np.zeros_like(root)
    if loc == XNEG:
        R[0, : S.shape[0]] = S @ root[0, : S.shape[0]]
    elif loc == XPOS:
        R[-1, : S.shape[0]] = S @ root[-1, : S.shape[0]]
    elif loc == YPOS:
        R[: S.shape[0], -1] = S @ root[: S.shape[0], -1]
    else:
        R[: S.shape[0], 0] = S @ root[: S.shape[0], 0]
    return R


class GMRESSolver2D:
    """GMRESSolver2D (pe/concat/gmres_solver2d.cpp:3-252): restarted GMRES(m) with classical Gram-Schmidt
    and Givens rotations on full root fields, absolute tolerance on ||r|| and |g_{j+1}|."""

    def __init__(self, m, tol, max_iter, pe_solve):
        self.m, self.tol, self.max_iter, self.pe_solve = m, tol, max_iter, pe_solve
        self.S = []  # (loc, matrix)
        self.res = []

    def afun(self, x):
        ft = np.zeros_like(x)
        for loc, S in self.S:
            ft = ft + schur_apply(loc, S, x)
        ft = self.pe_solve(ft)
        return x - ft

    def solve(self, b):
        m, tol = self.m, self.tol
        b = self.pe_solve(b)
        self.res = []
        x = b.copy()
        for _outer in range(self.max_iter):
            r = b - self.afun(x)
            beta = math.sqrt(float(np.dot(r.ravel(), r.ravel())))
            self.res.append(beta)
            if beta < tol:
                return x
            H = np.zeros((m + 1, m))
            cs = np.zeros(m)
            sn = np.zeros(m)
            g = np.zeros(m + 1)
            V = [r / beta]
            g[0] = beta
            j = 0
            while j < m:
                w = self.afun(V[j])
                for i in range(j + 1):
                    H[i, j] = float(np.dot(V[i].ravel(), w.ravel()))
                    w = w - H[i, j] * V[i]
                h = math.sqrt(float(np.dot(w.ravel(), w.ravel())))
                if h < 1e-12:
                    break
                H[j + 1, j] = h
                V.append(w / h)
                for i in range(j):
                    t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                    H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                    H[i, j] = t
                den = math.hypot(H[j, j], H[j + 1, j])
                cs[j] = H[j, j] / den
                sn[j] = H[j + 1, j] / den
                H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
                H[j + 1, j] = 0.0
                t = cs[j] * g[j]
                g[j + 1] = -sn[j] * g[j]
                g[j] = t
                if abs(g[j + 1]) < tol:
                    j += 1
                    break
                j += 1
            y = np.zeros(m)
            for i in range(j - 1, -1, -1):
                y[i] = g[i]
                for k in range(i + 1, j):
                    y[i] -= H[i, k] * y[k]
                y[i] /= H[i, i]
            for i in range(j):
                x = x + y[i] * V[i]
        return x


@dataclass
class Domain:
    nx: int
    ny: int
    hx: float
    hy: float
    bc: list = dc_field(default_factory=lambda: [D, D, D, D])  # faces not adjacented


@dataclass
class Tree:
    root: int
    children: dict  # domain -> list of (loc, child)
    parent: dict  # child -> (loc_of_parent_seen_from_child, parent)
    levels: list  # BFS levels, root first


def build_tree(n_domains: int, connections, root: int | None = None, faces=(XNEG, XPOS, YNEG, YPOS)) -> Tree:
    """Geometry2D::build_tree (geometry2d.cpp:165-176) with TreeUtils (geometry_tree.hpp:22-200); Geometry3D
    (geometry3d.cpp:151-160) builds its tree the same way over six faces."""
    adj = {i: {} for i in range(n_domains)}
    for a, loc, b in connections:
        adj[a][loc] = b
        adj[b][opposite(loc)] = a
    if root is None:
        if n_domains == 1:
            root = 0
        else:
            deg = {i: len(adj[i]) for i in adj}
            leaves = [i for i in sorted(adj) if deg[i] <= 1]
            remaining = n_domains
            while remaining > 2 and leaves:
                remaining -= len(leaves)
                nxt = []
                for lf in leaves:
                    for nb in adj[lf].values():
                        deg[nb] -= 1
                        if deg[nb] == 1:
                            nxt.append(nb)
                leaves = nxt
            root = min(leaves) if leaves else 0
    children = {i: [] for i in range(n_domains)}
    parent = {}

    def rec(cur, par):
        for loc in faces:
            nb = adj[cur].get(loc)
            if nb is None or nb == par:
                continue
            children[cur].append((loc, nb))
            parent[nb] = (opposite(loc), cur)
            rec(nb, cur)

    rec(root, None)
    levels, frontier = [], [root]
    while frontier:
        levels.append(frontier)
        frontier = [c for d in frontier for _, c in children[d]]
    return Tree(root, children, parent, levels)


class ConcatPoissonSolver2D:
    """ConcatPoissonSolver2D (pe/concat/concat_solver2d.cpp). domains[i].bc holds the boundary type of each
    face; adjacented faces are overridden from the connections (variable2d.cpp:25-45)."""

    def __init__(self, domains, connections, m=20, tol=1e-8, max_iter=100, root=None, schur=None):
        """schur: optional per-domain-index Schur matrices to use instead of building them by impulse
        solves (e.g. oracle/schur_closed_form.py for large leaves)."""
        self.domains = domains
        self.tree = build_tree(len(domains), connections, root)
        self.bc = []
        for i, d in enumerate(domains):
            b = list(d.bc)
            for a, loc, bb in connections:
                if a == i:
                    b[loc] = ADJ
                if bb == i:
                    b[opposite(loc)] = ADJ
            self.bc.append(b)
        self.m, self.tol, self.max_iter = m, tol, max_iter
        self.solvers = {}
        for lvl in reversed(self.tree.levels):  # construct_solver_map, concat_solver2d.cpp:88-99
            for d in lvl:
                dom = domains[d]
                ps = PoissonSolver2D(dom.nx, dom.ny, dom.hx, dom.hy, self.bc[d])
                if self.tree.children[d]:
                    g = GMRESSolver2D(m, tol, max_iter, ps.solve)
                    for loc, c in self.tree.children[d]:
                        cd_ = domains[c]
                        S = schur[c] if schur is not None and schur[c] is not None else None
                        g.S.append((loc, S if S is not None else schur_matrix(loc, cd_.nx, cd_.ny, self.solvers[c])))
                    self.solvers[d] = g.solve
                    self.gmres = g if d == self.tree.root else getattr(self, "gmres", None)
                else:
                    self.solvers[d] = ps.solve

    def boundary_assembly(self, fields, ghosts):
        """concat_solver2d.cpp:159-223. ghosts[i][face] = buffer values (or None = zero)."""
        for i, dom in enumerate(self.domains):
            f = fields[i]
            bt = self.bc[i]
            hx, hy = dom.hx, dom.hy

            def g(face):
                v = ghosts[i][face] if ghosts is not None and ghosts[i] is not None else None
                n = dom.ny if face in (XNEG, XPOS) else dom.nx
                return np.zeros(n) if v is None else np.asarray(v, dtype=np.float64)

            for face, coef in ((XNEG, -1.0 / hx / hx), (XPOS, -1.0 / hx / hx), (YNEG, -1.0 / hy / hy), (YPOS, -1.0 / hy / hy)):
                if bt[face] == D:
                    _edge_add(f, face, coef, g(face))
            for face, coef in ((XNEG, 1.0 / hx), (XPOS, -1.0 / hx), (YNEG, 1.0 / hy), (YPOS, -1.0 / hy)):
                if bt[face] == N:
                    _edge_add(f, face, coef, g(face))

    def solve(self, fields, ghosts=None):
        """ConcatPoissonSolver2D::solve, concat_solver2d.cpp:101-157. Returns the solution fields."""
        f = [np.array(x, dtype=np.float64, copy=True) for x in fields]
        self.boundary_assembly(f, ghosts)
        for i, dom in enumerate(self.domains):
            f[i] *= dom.hx * dom.hx
        T = self.tree
        temp = {}
        for lvl in reversed(T.levels[1:]):
            for d in lvl:
                temp[d] = f[d].copy()
                for loc, c in T.children[d]:
                    bond_add(temp[d], loc, -1.0, temp[c])
                    bond_add(f[d], loc, -1.0, temp[c])
            for d in lvl:
                temp[d] = self.solvers[d](temp[d])
        for loc, c in T.children[T.root]:
            bond_add(f[T.root], loc, -1.0, temp[c])
        f[T.root] = self.solvers[T.root](f[T.root])
        for lvl in T.levels[1:]:
            for d in lvl:
                ploc, par = T.parent[d]
                bond_add(f[d], ploc, -1.0, f[par])
            for d in lvl:
                f[d] = self.solvers[d](f[d])
        return f


def _edge_add(f, face, a, bound):
    """field2::{xneg,xpos,yneg,up}_bond_add(a, double*), field2.cpp:212-236."""
    if face == XNEG:
        f[0, :] += a * bound
    elif face == XPOS:
        f[-1, :] += a * bound
    elif face == YNEG:
        f[:, 0] += a * bound
    else:
        f[:, -1] += a * bound


def mock_solve(f):
    """The mock branch solver of case/validation/2d/gmres_reference.cpp:8-23."""
    nx, ny = f.shape
    i = np.arange(nx)[:, None]
    j = np.arange(ny)[None, :]
    return f * (i * ny + j + 1)


def composite_apply(domains, connections, bc, u):
    """The discrete composite operator the reference's block elimination inverts, in its hx^2-scaled form
    (concat_solver2d.cpp:101-157 with the rectangle operator of poisson_solver2d.cpp:46-51):
    (A u)_ij = u_{i-1,j} + u_{i+1,j} - 2u_ij + (hx/hy)^2 (u_{i,j-1} + u_{i,j+1} - 2u_ij), with ghost cells
    0 (Dirichlet), mirrored (Neumann), wrapped (periodic), and on Adjacented faces the neighbour's adjacent
    cells entering with coefficient 1 (bond_add(loc, -1, nb) moved to the left-hand side)."""
    nb = {(a, loc): b for a, loc, b in connections}
    nb.update({(b, opposite(loc)): a for a, loc, b in connections})
    out = []
    for d, dom in enumerate(domains):
        x = u[d]
        nx, ny = x.shape
        r2 = dom.hx * dom.hx / dom.hy / dom.hy

        def ghost(face):
            t = bc[d][face]
            if face == XNEG:
                own, wrap = x[0, :], x[nx - 1, :]
            elif face == XPOS:
                own, wrap = x[nx - 1, :], x[0, :]
            elif face == YNEG:
                own, wrap = x[:, 0], x[:, ny - 1]
            else:
                own, wrap = x[:, ny - 1], x[:, 0]
            if t == D:
                return np.zeros_like(own), 1.0
            if t == N:
                return own, 1.0
            if t == P:
                return wrap, 1.0
            o = u[nb[(d, face)]]
            edge = {XNEG: o[-1, :], XPOS: o[0, :], YNEG: o[:, -1], YPOS: o[:, 0]}[face]
            return edge, 0.0

        xm = np.vstack([ghost(XNEG)[0][None, :], x[:-1, :]])
        xp = np.vstack([x[1:, :], ghost(XPOS)[0][None, :]])
        gy0, sy0 = ghost(YNEG)
        gy1, sy1 = ghost(YPOS)
        ym = np.hstack([gy0[:, None], x[:, :-1]])
        yp = np.hstack([x[:, 1:], gy1[:, None]])
        lap = xm + xp - 2.0 * x + r2 * (yp + ym - 2.0 * x)
        # an Adjacented y face couples with coefficient 1, not (hx/hy)^2
        if sy0 == 0.0:
            lap[:, 0] += (1.0 - r2) * gy0
        if sy1 == 0.0:
            lap[:, -1] += (1.0 - r2) * gy1
        out.append(lap)
    return out


# ---------------------------------------------------------------------------------------------------
# 3D composite (ConcatPoissonSolver3D). Fields are (nx, ny, nz) arrays, value(i, j, k) = f[i, j, k]; a face
# plane is indexed as the reference's Schur matrices index it: x faces (j, k), y faces (i, k), z faces (i, j).

def _plane(f: np.ndarray, face: int, outer: bool) -> np.ndarray:
    """View of the boundary plane of f on `face` (outer=False: the layer at that face)."""
    nx, ny, nz = f.shape
    if face == XNEG:
        return f[0, :, :]
    if face == XPOS:
        return f[nx - 1, :, :]
    if face == YNEG:
        return f[:, 0, :]
    if face == YPOS:
        return f[:, ny - 1, :]
    if face == ZNEG:
        return f[:, :, 0]
    if face == ZPOS:
        return f[:, :, nz - 1]
    raise ValueError(face)


def bond_add3(f: np.ndarray, loc: int, a: float, nb: np.ndarray) -> None:
    """field3::bond_add(LocationType, a, const field3&) -- field3.cpp:306-375 (in place): the layer of f at
    `loc` gains a times the neighbour's layer on the opposite face."""
    _plane(f, loc, False)[...] += a * _plane(nb, opposite(loc), False)


def schur_matrix3(loc: int, shape, branch_solve) -> np.ndarray:
    """SchurMat3D_*::construct (schur_mat3d.cpp): column c = the branch's layer facing the node after a solve
    with a unit impulse at cell c of that layer (row / column index over the plane, row-major)."""
    face = opposite(loc)  # the branch's face toward the node
    t = np.zeros(shape)
    pl = _plane(t, face, False)
    cn = pl.size
    S = np.empty((cn, cn))
    for c in range(cn):
        t[...] = 0.0
        pl[np.unravel_index(c, pl.shape)] = 1.0
        u = branch_solve(t.copy())
        S[:, c] = _plane(u, face, False).reshape(-1)
    return S


def schur_apply3(loc: int, S: np.ndarray, x: np.ndarray) -> np.ndarray:
    """SchurMat3D_*::operator* (schur_mat3d.cpp): R zero except its layer at loc = S times x's layer there."""
    R = np.zeros_like(x)
    pl = _plane(x, loc, False)
    _plane(R, loc, False)[...] = (S @ pl.reshape(-1)).reshape(pl.shape)
    return R


class GMRESSolver3D:
    """GMRESSolver3D (pe/concat/gmres_solver3d.cpp:155-306): restarted GMRES(m) on full 3D fields for
    (I - A^-1 S) x = A^-1 b, modified Gram-Schmidt, Givens rotations, absolute tolerance on ||r|| (restart test)
    and |g_{j+1}| (inner test)."""

    def __init__(self, m, tol, max_iter, pe_solve):
        self.m, self.tol, self.max_iter, self.pe_solve = m, tol, max_iter, pe_solve
        self.S = []  # (loc, matrix)
        self.res = []

    def afun(self, x):
        ft = np.zeros_like(x)
        for loc, S in self.S:
            ft = ft + schur_apply3(loc, S, x)
        ft = self.pe_solve(ft)
        return x - ft

    def solve(self, b):
        m, tol = self.m, self.tol
        b = self.pe_solve(b)
        self.res = []
        x = b.copy()
        for _outer in range(self.max_iter):
            r = b - self.afun(x)
            beta = math.sqrt(float(np.dot(r.ravel(), r.ravel())))
            self.res.append(beta)
            if beta < tol:
                return x
            H = np.zeros((m + 1, m))
            cs = np.zeros(m)
            sn = np.zeros(m)
            g = np.zeros(m + 1)
            V = [r * (1.0 / beta)]
            g[0] = beta
            j = 0
            while j < m:
                w = self.afun(V[j])
                for i in range(j + 1):
                    H[i, j] = float(np.dot(V[i].ravel(), w.ravel()))
                    w = w - H[i, j] * V[i]
                h = math.sqrt(float(np.dot(w.ravel(), w.ravel())))
                if h < 1e-12:
                    break
                H[j + 1, j] = h
                V.append(w * (1.0 / h))
                for i in range(j):
                    t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                    H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                    H[i, j] = t
                den = math.hypot(H[j, j], H[j + 1, j])
                cs[j] = H[j, j] / den
                sn[j] = H[j + 1, j] / den
                H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
                H[j + 1, j] = 0.0
                t = cs[j] * g[j]
                g[j + 1] = -sn[j] * g[j]
                g[j] = t
                if abs(g[j + 1]) < tol:
                    j += 1
                    break
                j += 1
            y = np.zeros(m)
            for i in range(j - 1, -1, -1):
                y[i] = g[i]
                for k in range(i + 1, j):
                    y[i] -= H[i, k] * y[k]
                y[i] /= H[i, i]
            for i in range(j):
                x = x + y[i] * V[i]
        return x


@dataclass
class Domain3:
    nx: int
    ny: int
    nz: int
    hx: float
    hy: float
    hz: float
    bc: list = dc_field(default_factory=lambda: [D] * 6)  # faces not adjacented


class ConcatPoissonSolver3D:
    """ConcatPoissonSolver3D (pe/concat/concat_solver3d.cpp:5-247). domains[i].bc holds the boundary type of
    each of the six faces; adjacented faces are overridden from the connections."""

    def __init__(self, domains, connections, m=20, tol=1e-8, max_iter=100, root=None):
        self.domains = domains
        self.tree = build_tree(len(domains), connections, root, faces=(XNEG, XPOS, YNEG, YPOS, ZNEG, ZPOS))
        self.bc = []
        for i, d in enumerate(domains):
            b = list(d.bc)
            for a, loc, bb in connections:
                if a == i:
                    b[loc] = ADJ
                if bb == i:
                    b[opposite(loc)] = ADJ
            self.bc.append(b)
        self.solvers = {}
        for lvl in reversed(self.tree.levels):  # construct_solver_map, concat_solver3d.cpp:72-98
            for d in lvl:
                dom = domains[d]
                ps = PoissonSolver3D(dom.nx, dom.ny, dom.nz, dom.hx, dom.hy, dom.hz, self.bc[d])
                if self.tree.children[d]:
                    g = GMRESSolver3D(m, tol, max_iter, ps.solve)
                    for loc, c in self.tree.children[d]:
                        cd_ = domains[c]
                        g.S.append((loc, schur_matrix3(loc, (cd_.nx, cd_.ny, cd_.nz), self.solvers[c])))
                    self.solvers[d] = g.solve
                else:
                    self.solvers[d] = ps.solve

    def boundary_assembly(self, fields, ghosts):
        """concat_solver3d.cpp:159-247. ghosts[i][face]: the face's buffer values ((ny, nz), (nx, nz) or
        (nx, ny); None = zero)."""
        for i, dom in enumerate(self.domains):
            f, bt = fields[i], self.bc[i]
            hs = (dom.hx, dom.hx, dom.hy, dom.hy, dom.hz, dom.hz)

            def g(face):
                v = ghosts[i][face] if ghosts is not None and ghosts[i] is not None else None
                return 0.0 if v is None else np.asarray(v, dtype=np.float64)

            for face in range(6):  # Dirichlet faces first, then Neumann faces, as the reference adds them
                if bt[face] == D:
                    _plane(f, face, False)[...] += (-1.0 / hs[face] / hs[face]) * g(face)
            for face in range(6):
                if bt[face] == N:
                    _plane(f, face, False)[...] += ((1.0 if face % 2 == 0 else -1.0) / hs[face]) * g(face)

    def solve(self, fields, ghosts=None):
        """ConcatPoissonSolver3D::solve, concat_solver3d.cpp:100-157. Returns the solution fields."""
        f = [np.array(x, dtype=np.float64, copy=True) for x in fields]
        self.boundary_assembly(f, ghosts)
        for i, dom in enumerate(self.domains):
            f[i] *= dom.hx * dom.hx
        T = self.tree
        temp = {}
        for lvl in reversed(T.levels[1:]):
            for d in lvl:
                temp[d] = f[d].copy()
                for loc, c in T.children[d]:
                    bond_add3(temp[d], loc, -1.0, temp[c])
                    bond_add3(f[d], loc, -1.0, temp[c])
            for d in lvl:
                temp[d] = self.solvers[d](temp[d])
        for loc, c in T.children[T.root]:
            bond_add3(f[T.root], loc, -1.0, temp[c])
        f[T.root] = self.solvers[T.root](f[T.root])
        for lvl in T.levels[1:]:
            for d in lvl:
                ploc, par = T.parent[d]
                bond_add3(f[d], ploc, -1.0, f[par])
            for d in lvl:
                f[d] = self.solvers[d](f[d])
        return f

