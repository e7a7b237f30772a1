"""ctypes binding to oracle/_ref/libfpref.so: the reference's own serial 2D sources built for CPU.

TEST INFRASTRUCTURE. Callers: tests/golden/make_golden.py (fixture generation), tests/ (pinning the numpy
restatement when the library is present) and bench.py's CPU reference arm. See oracle/ref_harness.cpp
for the reference routine behind each entry point.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfpref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.fpref_transform.argtypes = [ctypes.c_int] * 5 + [vp, vp]
        L.fpref_transform.restype = ctypes.c_int
        L.fpref_poisson2d_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, vp, vp,
                                            ctypes.c_int, dp]
        L.fpref_poisson2d_solve.restype = ctypes.c_int
        L.fpref_poisson3d_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, vp, vp, ctypes.c_int, dp]
        L.fpref_poisson3d_solve.restype = ctypes.c_int
        L.fpref_concat_create.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, vp]
        L.fpref_concat_create.restype = vp
        L.fpref_concat_construct_seconds.argtypes = [vp]
        L.fpref_concat_construct_seconds.restype = ctypes.c_double
        L.fpref_concat_tree.argtypes = [vp, ip, vp]
        L.fpref_concat_tree.restype = ctypes.c_int
        L.fpref_concat_solve.argtypes = [vp, vp, vp, vp, ctypes.c_int]
        L.fpref_concat_solve.restype = ctypes.c_double
        L.fpref_concat_destroy.argtypes = [vp]
        L.fpref_concat3d_create.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp,
                                            ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.fpref_concat3d_create.restype = vp
        L.fpref_concat3d_tree.argtypes = [vp, ip, vp]
        L.fpref_concat3d_tree.restype = ctypes.c_int
        L.fpref_concat3d_solve.argtypes = [vp, vp, vp, vp]
        L.fpref_concat3d_solve.restype = ctypes.c_double
        L.fpref_concat3d_destroy.argtypes = [vp]
        L.fpref_gmres_mock.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_int, vp]
        L.fpref_schur_mock.argtypes = [ctypes.c_int] * 5 + [vp, vp]
        L.fpref_add_random.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp]
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def transform(bn: int, bp: int, f: np.ndarray, inverse: bool = False) -> np.ndarray:
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.empty_like(f)
    rc = lib().fpref_transform(bn, bp, f.shape[0], f.shape[1], int(inverse), _ptr(f), _ptr(out))
    if rc:
        raise ValueError("unsupported boundary pair")
    return out


def poisson2d_solve(f: np.ndarray, hx: float, hy: float, bc, repeats: int = 1):
    f = np.array(f, dtype=np.float64, copy=True, order="C")
    bca = np.asarray(bc, dtype=np.int32)
    t = ctypes.c_double(0.0)
    lib().fpref_poisson2d_solve(f.shape[0], f.shape[1], float(hx), float(hy), _ptr(bca), _ptr(f), repeats,
                                ctypes.byref(t))
    return f, t.value


def poisson3d_solve(f: np.ndarray, hx: float, hy: float, hz: float, bc, repeats: int = 1):
    """The reference's PoissonSolver3D(nx, ny, nz, hx, hy, hz, bc[6]).solve on a copy of f (nx, ny, nz)."""
    f = np.array(f, dtype=np.float64, copy=True, order="C")
    bca = np.asarray(bc, dtype=np.int32)
    t = ctypes.c_double(0.0)
    nx, ny, nz = f.shape
    lib().fpref_poisson3d_solve(nx, ny, nz, float(hx), float(hy), float(hz), _ptr(bca), _ptr(f), repeats,
                                ctypes.byref(t))
    return f, t.value


class ConcatCase:
    """Geometry + Variable2D + ConcatPoissonSolver2D built by the reference (constructor timed)."""

    def __init__(self, nx, ny, lx, ly, connections, bc, m=20, tol=1e-8, max_iter=100, schur=None):
        nd = len(nx)
        self._keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt))
            self._keep.append(a)
            return _ptr(a)

        ca = [c[0] for c in connections]
        cd = [c[1] for c in connections]
        cb = [c[2] for c in connections]
        S_ptrs = None
        if schur is not None:
            arrs = [None if s is None else np.ascontiguousarray(s, dtype=np.float64) for s in schur]
            self._keep.extend([a for a in arrs if a is not None])
            S_ptrs = (ctypes.c_void_p * nd)(*[None if a is None else a.ctypes.data for a in arrs])
        self.h = lib().fpref_concat_create(nd, arr(nx, np.int32), arr(ny, np.int32), arr(lx, np.float64),
                                           arr(ly, np.float64), len(connections), arr(ca, np.int32),
                                           arr(cd, np.int32), arr(cb, np.int32),
                                           arr(np.asarray(bc).ravel(), np.int32), m, float(tol), max_iter,
                                           S_ptrs)
        if not self.h:
            raise RuntimeError("reference case construction failed")
        self.nd = nd
        self.shapes = list(zip(nx, ny))
        self.construct_seconds = lib().fpref_concat_construct_seconds(self.h)

    def tree(self):
        root = ctypes.c_int(0)
        lv = np.zeros(self.nd, dtype=np.int32)
        lib().fpref_concat_tree(self.h, ctypes.byref(root), _ptr(lv))
        return root.value, lv

    def solve(self, rhs, ghosts=None, repeats: int = 1):
        rhs = [np.ascontiguousarray(r, dtype=np.float64) for r in rhs]
        outs = [np.empty_like(r) for r in rhs]
        rp = (ctypes.c_void_p * self.nd)(*[r.ctypes.data for r in rhs])
        op = (ctypes.c_void_p * self.nd)(*[o.ctypes.data for o in outs])
        gp = None
        if ghosts is not None:
            gl = []
            for i in range(self.nd):
                for f in range(4):
                    g = None if ghosts[i] is None else ghosts[i][f]
                    if g is not None:
                        g = np.ascontiguousarray(g, dtype=np.float64)
                        self._keep.append(g)
                    gl.append(None if g is None else g.ctypes.data)
            gp = (ctypes.c_void_p * (4 * self.nd))(*gl)
        t = lib().fpref_concat_solve(self.h, rp, gp, op, repeats)
        return outs, t

    def __del__(self):
        if getattr(self, "h", None):
            lib().fpref_concat_destroy(self.h)
            self.h = None


class Concat3DCase:
    """Geometry3D + Variable3D + ConcatPoissonSolver3D built by the reference (pe/concat/concat_solver3d.cpp).
    Domains (nx, ny, nz, lx, ly, lz) per index, connections (a, face of a, b), bc: 6 per domain (faces x-, x+,
    y-, y+, z-, z+; ignored where adjacented)."""

    def __init__(self, nx, ny, nz, lx, ly, lz, connections, bc, m=20, tol=1e-8, max_iter=100):
        nd = len(nx)
        self._keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt))
            self._keep.append(a)
            return _ptr(a)

        self.h = lib().fpref_concat3d_create(nd, arr(nx, np.int32), arr(ny, np.int32), arr(nz, np.int32),
                                             arr(lx, np.float64), arr(ly, np.float64), arr(lz, np.float64),
                                             len(connections), arr([c[0] for c in connections], np.int32),
                                             arr([c[1] for c in connections], np.int32),
                                             arr([c[2] for c in connections], np.int32),
                                             arr(np.asarray(bc).ravel(), np.int32), m, float(tol), max_iter)
        if not self.h:
            raise RuntimeError("reference case construction failed")
        self.nd = nd

    def tree(self):
        root = ctypes.c_int(0)
        lv = np.zeros(self.nd, dtype=np.int32)
        lib().fpref_concat3d_tree(self.h, ctypes.byref(root), _ptr(lv))
        return root.value, lv

    def solve(self, rhs, ghosts=None):
        """rhs: per domain (nx, ny, nz) arrays; ghosts: None or per domain 6 arrays / None (x faces (ny, nz),
        y faces (nx, nz), z faces (nx, ny)). Returns the solution fields and the solve time."""
        rhs = [np.ascontiguousarray(r, dtype=np.float64) for r in rhs]
        outs = [np.empty_like(r) for r in rhs]
        rp = (ctypes.c_void_p * self.nd)(*[r.ctypes.data for r in rhs])
        op = (ctypes.c_void_p * self.nd)(*[o.ctypes.data for o in outs])
        gp = None
        if ghosts is not None:
            gl = []
            for i in range(self.nd):
                for f in range(6):
                    g = None if ghosts[i] is None else ghosts[i][f]
                    if g is not None:
                        g = np.ascontiguousarray(g, dtype=np.float64)
                        self._keep.append(g)
                    gl.append(None if g is None else g.ctypes.data)
            gp = (ctypes.c_void_p * (6 * self.nd))(*gl)
        t = lib().fpref_concat3d_solve(self.h, rp, gp, op)
        return outs, t

    def __del__(self):
        if getattr(self, "h", None):
            lib().fpref_concat3d_destroy(self.h)
            self.h = None


def gmres_mock(loc, nx, ny, neighbor_n, m, tol, max_iter):
    out = np.empty((nx, ny))
    lib().fpref_gmres_mock(loc, nx, ny, neighbor_n, m, float(tol), max_iter, _ptr(out))
    return out


def schur_mock(loc, bnx, bny, nx, ny):
    cn = bny if loc in (0, 1) else bnx
    S = np.empty((cn, cn))
    prod = np.empty((nx, ny))
    lib().fpref_schur_mock(loc, bnx, bny, nx, ny, _ptr(S), _ptr(prod))
    return S, prod


def add_random(f: np.ndarray, lo: float, hi: float, seed: int) -> np.ndarray:
    """The reference's add_random_number on a copy of f (interior cells only)."""
    f = np.array(f, dtype=np.float64, copy=True, order="C")
    lib().fpref_add_random(f.shape[0], f.shape[1], float(lo), float(hi), int(seed), _ptr(f))
    return f
