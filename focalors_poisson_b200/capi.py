"""ctypes binding of libfpb200.so (include/fp_capi.h).

The library is the only compute path: if it is missing or no CUDA device is present every call raises
(there is no CPU fallback). Arrays may be numpy (host, synchronous) or torch CUDA tensors (device,
queued on torch's current stream).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfpb200.so")

FP_DEVICE, FP_SYNC = 1, 2
FP_F64, FP_F32 = 0, 1
STATUS = {0: "FP_OK", 1: "FP_ERR_INVALID", 2: "FP_ERR_CUDA", 3: "FP_ERR_UNSUPPORTED", 4: "FP_ERR_NOT_CONVERGED",
          5: "FP_ERR_NAN", 6: "FP_ERR_NOMEM"}

# Every symbol include/fp_capi.h declares, with its ctypes signature.
_vp, _i, _d, _ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
SIGNATURES = {
    "fp_last_error": ([], ctypes.c_char_p),
    "fp_launch_count": ([], ctypes.c_longlong),
    "fp_transform_f64": ([_i, _i, _i, _i, _i, _vp, _vp, _i, _vp], _i),
    "fp_transform_f32": ([_i, _i, _i, _i, _i, _vp, _vp, _i, _vp], _i),
    "fp_rect_create": ([_i, _i, _d, _d, _vp, _i, _vp], _i),
    "fp_rect_solve_f64": ([_vp, _vp, _ll, _i, _vp], _i),
    "fp_rect_chase_f64": ([_vp, _vp, _ll, _i, _vp], _i),
    "fp_field_fill": ([_vp, _i, _i, _d, _d, _d, _d, _i, _vp, _i, _i, _vp], _i),
    "fp_buffer_fill": ([_vp, _i, _i, _i, _d, _d, _d, _d, _i, _vp, _i, _vp], _i),
    "fp_rect_solve_f32": ([_vp, _vp, _ll, _i, _vp], _i),
    "fp_rect3d_create": ([_i, _i, _i, _d, _d, _d, _vp, _vp], _i),
    "fp_rect3d_solve_f64": ([_vp, _vp, _ll, _i, _vp], _i),
    "fp_rect3d_destroy": ([_vp], _i),
    "fp_rect_destroy": ([_vp], _i),
    "fp_rect_solve_f64_noalloc": ([_vp, _vp, _ll, _vp], _i),
    "fp_composite_create": ([_vp, _i, _d, _i, _i, _vp], _i),
    "fp_composite_set_parameter": ([_vp, _i, _d, _i], _i),
    "fp_composite_solve_f64": ([_vp, _vp, _vp, _i, _vp, _vp], _i),
    "fp_composite_solve_f32ir": ([_vp, _vp, _vp, _i, _vp, _d, _i, _vp], _i),
    "fp_composite_adjoint_f64": ([_vp, _vp, _i, _vp, _vp], _i),
    "fp_composite_adjoint_f32ir": ([_vp, _vp, _i, _vp, _d, _i, _vp], _i),
    "fp_composite3d_create": ([_vp, _i, _d, _i, _vp], _i),
    "fp_composite3d_set_parameter": ([_vp, _i, _d, _i], _i),
    "fp_composite3d_solve_f64": ([_vp, _vp, _vp, _i, _vp, _vp], _i),
    "fp_composite3d_tree": ([_vp, _vp, _vp], _i),
    "fp_composite3d_destroy": ([_vp], _i),
    "fp_composite_part_create": ([_vp, _i, _d, _i, _i, _i, _vp, _vp], _i),
    "fp_composite_part_schur": ([_vp, _i, _vp, _vp], _i),
    "fp_composite_set_external_schur": ([_vp, _i, _vp], _i),
    "fp_composite_part_upward": ([_vp, _vp, _vp, _i, _vp, _vp, _vp], _i),
    "fp_composite_part_downward": ([_vp, _vp, _i, _vp, _vp, _vp], _i),
    "fp_composite_root_solve": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "fp_composite_solve_async": ([_vp, _vp, _vp, _vp, _i, _d, _i, _vp], _i),
    "fp_composite_wait": ([_vp, _i, _vp], _i),
    "fp_composite_residual": ([_vp, _vp, _vp, _vp, _vp, _vp], _i),
    "fp_composite_tree": ([_vp, _vp, _vp], _i),
    "fp_composite_destroy": ([_vp], _i),
    "fp_batch_create": ([_vp, _i, _i, _vp], _i),
    "fp_batch_solve": ([_vp, _vp, _vp, _i, _vp, _i], _i),
    "fp_batch_residuals": ([_vp, _vp, _vp, _vp, _vp, _vp], _i),
    "fp_batch_info": ([_vp, _vp, _vp, _vp, _vp], _i),
    "fp_batch_destroy": ([_vp], _i),
}
FP_GMRES_FULLFIELD, FP_CHECK_CONVERGENCE, FP_NO_INTERFACE_INVERSE, FP_IR_INNER_F64 = 4, 8, 16, 32
FP_BATCH_F32, FP_BATCH_NO_AUTOTUNE, FP_BATCH_GRAPH, FP_NO_SPECTRAL, FP_IR_FIRST_F64 = 64, 128, 256, 512, 1024
FP_FORM_F64, FP_FORM_F64IR, FP_FORM_F32IR, FP_FORM_MIXEDIR = 0, 1, 2, 3
FORMS = {"f64": FP_FORM_F64, "f64ir": FP_FORM_F64IR, "f32ir": FP_FORM_F32IR, "mixedir": FP_FORM_MIXEDIR}


class Geometry(ctypes.Structure):
    """struct fp_geometry"""

    _fields_ = [("n_domains", ctypes.c_int), ("nx", _vp), ("ny", _vp), ("hx", _vp), ("hy", _vp), ("bc", _vp),
                ("n_connections", ctypes.c_int), ("connections", _vp), ("root", ctypes.c_int)]


class Geometry3(ctypes.Structure):
    """struct fp_geometry3"""

    _fields_ = [("n_domains", ctypes.c_int), ("nx", _vp), ("ny", _vp), ("nz", _vp), ("hx", _vp), ("hy", _vp),
                ("hz", _vp), ("bc", _vp), ("n_connections", ctypes.c_int), ("connections", _vp),
                ("root", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    """struct fp_solve_info"""

    _fields_ = [("gmres_iterations", ctypes.c_int), ("gmres_restarts", ctypes.c_int),
                ("gmres_residual", ctypes.c_double), ("converged", ctypes.c_int), ("refinements", ctypes.c_int),
                ("rel_change", ctypes.c_double)]

_lib = None


class FpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads libfpb200.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m focalors_poisson_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int, allow=()):
    if rc != 0 and rc not in allow:
        raise FpError(rc, lib().fp_last_error().decode())
    return rc


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _args(x, want):
    """(pointer, flags, stream, keepalive) for a numpy array or a torch CUDA tensor of dtype `want`."""
    if _is_torch(x):
        import torch

        tdt = torch.float64 if want == np.float64 else torch.float32
        if not x.is_cuda or x.dtype != tdt or not x.is_contiguous():
            raise TypeError(f"expected a contiguous CUDA {tdt} tensor")
        return ctypes.c_void_p(x.data_ptr()), FP_DEVICE, _stream(), x
    a = np.ascontiguousarray(x, dtype=want)
    return ctypes.c_void_p(a.ctypes.data), 0, None, a


def transform(bc_yneg: int, bc_ypos: int, f, inverse: bool = False, out=None):
    """PoissonFFT2D_* transform (forward) or transform_transpose (inverse) of an (nx, ny) field."""
    want = np.float32 if (getattr(f, "dtype", None) in (np.float32,) or str(getattr(f, "dtype", "")) == "torch.float32") else np.float64
    nx, ny = f.shape[-2], f.shape[-1]
    rows = int(np.prod(f.shape[:-1]))
    if out is None:
        out = f.clone() if _is_torch(f) else np.empty(f.shape, dtype=want)
    p_in, flags, stream, keep_in = _args(f, want)
    p_out, _, _, keep_out = _args(out, want)
    fn = lib().fp_transform_f32 if want == np.float32 else lib().fp_transform_f64
    check(fn(bc_yneg, bc_ypos, rows, ny, int(inverse), p_in, p_out, flags, stream))
    if not _is_torch(out) and keep_out is not out:
        out[...] = keep_out
    return out


class Rect:
    """PoissonSolver2D(nx, ny, hx, hy, bc) on the GPU: solve() works in place on (…, nx, ny) arrays."""

    def __init__(self, nx, ny, hx, hy, bc, precision=FP_F64):
        self.nx, self.ny, self.precision = nx, ny, precision
        h = ctypes.c_void_p()
        bca = (ctypes.c_int * 4)(*[int(b) for b in bc])
        check(lib().fp_rect_create(nx, ny, float(hx), float(hy), bca, precision, ctypes.byref(h)))
        self.h = h

    def solve(self, f):
        want = np.float32 if self.precision == FP_F32 else np.float64
        if f.shape[-2:] != (self.nx, self.ny):
            raise ValueError("field shape does not match the solver")
        batch = int(np.prod(f.shape[:-2])) if len(f.shape) > 2 else 1
        p, flags, stream, keep = _args(f, want)
        fn = lib().fp_rect_solve_f32 if want == np.float32 else lib().fp_rect_solve_f64
        check(fn(self.h, p, batch, flags, stream))
        if not _is_torch(f) and keep is not f:
            f[...] = keep
        return f

    def chase(self, f):
        """The chasing step alone (ChasingMethod2D::chasing) on fields already in transformed space; FP64."""
        if self.precision != FP_F64 or f.shape[-2:] != (self.nx, self.ny):
            raise ValueError("chase needs an FP64 solver and fields of its shape")
        batch = int(np.prod(f.shape[:-2])) if len(f.shape) > 2 else 1
        p, flags, stream, keep = _args(f, np.float64)
        check(lib().fp_rect_chase_f64(self.h, p, batch, flags, stream))
        if not _is_torch(f) and keep is not f:
            f[...] = keep
        return f

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_rect_destroy(self.h)
            self.h = None


class Rect3D:
    """PoissonSolver3D(nx, ny, nz, hx, hy, hz, bc[6]) on the GPU: solve() works in place on (…, nx, ny, nz)
    float64 arrays (z contiguous, the reference's field3 layout)."""

    def __init__(self, nx, ny, nz, hx, hy, hz, bc):
        self.shape = (nx, ny, nz)
        h = ctypes.c_void_p()
        bca = (ctypes.c_int * 6)(*[int(b) for b in bc])
        check(lib().fp_rect3d_create(nx, ny, nz, float(hx), float(hy), float(hz), bca, ctypes.byref(h)))
        self.h = h

    def solve(self, f):
        if tuple(f.shape[-3:]) != self.shape:
            raise ValueError("field shape does not match the solver")
        batch = int(np.prod(f.shape[:-3])) if len(f.shape) > 3 else 1
        p, flags, stream, keep = _args(f, np.float64)
        check(lib().fp_rect3d_solve_f64(self.h, p, batch, flags, stream))
        if not _is_torch(f) and keep is not f:
            f[...] = keep
        return f

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_rect3d_destroy(self.h)
            self.h = None


class Composite3D:
    """ConcatPoissonSolver3D on the GPU for a tree of boxes.

    domains: [(nx, ny, nz, hx, hy, hz)], connections: [(a, face of a, b)] (faces 0..5: x-, x+, y-, y+, z-, z+),
    bc: 6 boundary types per domain (ignored on connected faces)."""

    def __init__(self, domains, connections, bc, m=20, tol=1e-8, max_iter=100, root=-1):
        nd = len(domains)
        self.nd = nd
        self.shapes = [(int(d[0]), int(d[1]), int(d[2])) for d in domains]
        cols = list(zip(*domains))
        self._arr = dict(nx=np.ascontiguousarray(cols[0], dtype=np.int32),
                         ny=np.ascontiguousarray(cols[1], dtype=np.int32),
                         nz=np.ascontiguousarray(cols[2], dtype=np.int32),
                         hx=np.ascontiguousarray(cols[3], dtype=np.float64),
                         hy=np.ascontiguousarray(cols[4], dtype=np.float64),
                         hz=np.ascontiguousarray(cols[5], dtype=np.float64),
                         bc=np.ascontiguousarray(np.asarray(bc, dtype=np.int32).reshape(-1)),
                         conn=np.ascontiguousarray(np.asarray(connections, dtype=np.int32).reshape(-1)))
        a = self._arr
        g = Geometry3(nd, a["nx"].ctypes.data, a["ny"].ctypes.data, a["nz"].ctypes.data, a["hx"].ctypes.data,
                      a["hy"].ctypes.data, a["hz"].ctypes.data, a["bc"].ctypes.data, len(connections),
                      a["conn"].ctypes.data if len(connections) else None, int(root))
        h = ctypes.c_void_p()
        check(lib().fp_composite3d_create(ctypes.byref(g), int(m), float(tol), int(max_iter), ctypes.byref(h)))
        self.h = h

    def set_parameter(self, m, tol, max_iter):
        check(lib().fp_composite3d_set_parameter(self.h, int(m), float(tol), int(max_iter)))

    def tree(self):
        root = ctypes.c_int(0)
        lv = np.zeros(self.nd, dtype=np.int32)
        check(lib().fp_composite3d_tree(self.h, ctypes.byref(root), lv.ctypes.data))
        return root.value, lv

    def solve(self, fields, ghosts=None, check_convergence=False):
        """ConcatPoissonSolver3D::solve in place. fields: per domain (nx, ny, nz) float64 numpy arrays (host) or
        CUDA tensors (device); ghosts: None or per domain 6 arrays / None (x faces (ny, nz), y faces (nx, nz),
        z faces (nx, ny)), on the same side as the fields."""
        if len(fields) != self.nd:
            raise ValueError("one field per domain expected")
        keep, ptrs, flags, stream = [], [], 0, None
        for f, shp in zip(fields, self.shapes):
            if tuple(f.shape) != shp:
                raise ValueError(f"field shape {tuple(f.shape)} != domain shape {shp}")
            p, fl, st, k = _args(f, np.float64)
            if not _is_torch(f) and k is not f:
                raise TypeError("host fields must be contiguous float64 numpy arrays (solved in place)")
            flags |= fl
            stream = st if st is not None else stream
            keep.append(k)
            ptrs.append(p.value)
        gp = None
        if ghosts is not None:
            gl = []
            for d in range(self.nd):
                for face in range(6):
                    gv = None if ghosts[d] is None else ghosts[d][face]
                    if gv is None:
                        gl.append(None)
                        continue
                    p, _, _, k = _args(gv, np.float64)
                    keep.append(k)
                    gl.append(p.value)
            gp = (ctypes.c_void_p * (6 * self.nd))(*gl)
        info = SolveInfo()
        if check_convergence:
            flags |= FP_CHECK_CONVERGENCE
        check(lib().fp_composite3d_solve_f64(self.h, (ctypes.c_void_p * self.nd)(*ptrs), gp, flags, stream,
                                             ctypes.byref(info)))
        return Composite._info(info)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_composite3d_destroy(self.h)
            self.h = None


def _cuda_ptrs(tensors, what):
    ptrs = []
    for t in tensors:
        if t is None:
            ptrs.append(None)
            continue
        if not _is_torch(t) or not t.is_cuda or not t.is_contiguous() or str(t.dtype) != "torch.float64":
            raise TypeError(f"{what}: contiguous float64 CUDA tensors expected")
        ptrs.append(t.data_ptr())
    return (ctypes.c_void_p * max(1, len(ptrs)))(*ptrs)


class CompositePart:
    """One part of a subtree decomposition of the composite solve (fp_composite_part_*): a subtree part
    (geometry of the subtree, its root's face toward the root domain Adjacented, ext_faces empty) or the root
    part (the root domain alone, ext_faces = the faces of its children in other parts, increasing). All
    arrays are float64 CUDA tensors; work is queued on torch's current stream."""

    def __init__(self, geo, m=20, tol=1e-8, max_iter=100, root=-1, ext_faces=()):
        nd = len(geo.nx)
        self.nd = nd
        self.shapes = [(int(a), int(b)) for a, b in zip(geo.nx, geo.ny)]
        self._arr = dict(
            nx=np.ascontiguousarray(geo.nx, dtype=np.int32), ny=np.ascontiguousarray(geo.ny, dtype=np.int32),
            hx=np.ascontiguousarray(geo.hx, dtype=np.float64), hy=np.ascontiguousarray(geo.hy, dtype=np.float64),
            bc=np.ascontiguousarray(np.asarray(geo.bc, dtype=np.int32).reshape(-1)),
            conn=np.ascontiguousarray(np.asarray(geo.connections, dtype=np.int32).reshape(-1)),
            ext=np.ascontiguousarray(np.asarray(list(ext_faces), dtype=np.int32)))
        a = self._arr
        g = Geometry(nd, a["nx"].ctypes.data, a["ny"].ctypes.data, a["hx"].ctypes.data, a["hy"].ctypes.data,
                     a["bc"].ctypes.data, len(geo.connections), a["conn"].ctypes.data if len(geo.connections) else None,
                     int(root))
        h = ctypes.c_void_p()
        check(lib().fp_composite_part_create(ctypes.byref(g), int(m), float(tol), int(max_iter), 0, len(ext_faces),
                                             a["ext"].ctypes.data if len(ext_faces) else None, ctypes.byref(h)))
        self.h = h

    @staticmethod
    def _info(info):
        return Composite._info(info)

    def schur(self, face, S):
        check(lib().fp_composite_part_schur(self.h, int(face), _cuda_ptrs([S], "S")[0], _stream()))

    def set_external_schur(self, k, S):
        check(lib().fp_composite_set_external_schur(self.h, int(k), _cuda_ptrs([S], "S")[0]))

    def _ghosts(self, ghosts):
        if ghosts is None:
            return None
        return _cuda_ptrs([None if ghosts[d] is None else ghosts[d][f] for d in range(self.nd) for f in range(4)],
                          "ghosts")

    def upward(self, fields, ghosts, face, edge_out):
        info = SolveInfo()
        check(lib().fp_composite_part_upward(self.h, _cuda_ptrs(fields, "fields"), self._ghosts(ghosts), int(face),
                                             _cuda_ptrs([edge_out], "edge")[0], _stream(), ctypes.byref(info)))
        return self._info(info)

    def downward(self, fields, face, parent_edge):
        info = SolveInfo()
        check(lib().fp_composite_part_downward(self.h, _cuda_ptrs(fields, "fields"), int(face),
                                               _cuda_ptrs([parent_edge], "edge")[0], _stream(), ctypes.byref(info)))
        return self._info(info)

    def root_solve(self, fields, ghosts, child_edges, edges_out):
        info = SolveInfo()
        check(lib().fp_composite_root_solve(self.h, _cuda_ptrs(fields, "fields"), self._ghosts(ghosts),
                                            _cuda_ptrs(child_edges, "child edges"), _cuda_ptrs(edges_out, "edges"),
                                            _stream(), ctypes.byref(info)))
        return self._info(info)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_composite_destroy(self.h)
            self.h = None


class Composite:
    """ConcatPoissonSolver2D on the GPU for a tree of rectangles.

    geo: any object with nx, ny, hx, hy (per domain lists), bc (4 faces per domain) and connections
    [(a, face of a, b)] -- e.g. focalors_poisson_b200.workloads.Geometry.
    """

    def __init__(self, geo, m=20, tol=1e-8, max_iter=100, root=-1, fullfield=False, interface_inverse=True,
                 spectral=True):
        nd = len(geo.nx)
        self.nd = nd
        self.shapes = [(int(a), int(b)) for a, b in zip(geo.nx, geo.ny)]
        self._arr = dict(
            nx=np.ascontiguousarray(geo.nx, dtype=np.int32), ny=np.ascontiguousarray(geo.ny, dtype=np.int32),
            hx=np.ascontiguousarray(geo.hx, dtype=np.float64), hy=np.ascontiguousarray(geo.hy, dtype=np.float64),
            bc=np.ascontiguousarray(np.asarray(geo.bc, dtype=np.int32).reshape(-1)),
            conn=np.ascontiguousarray(np.asarray(geo.connections, dtype=np.int32).reshape(-1)))
        a = self._arr
        g = Geometry(nd, a["nx"].ctypes.data, a["ny"].ctypes.data, a["hx"].ctypes.data, a["hy"].ctypes.data,
                     a["bc"].ctypes.data, len(geo.connections), a["conn"].ctypes.data if len(geo.connections) else None,
                     int(root))
        h = ctypes.c_void_p()
        flags = (FP_GMRES_FULLFIELD if fullfield else 0) | (0 if interface_inverse else FP_NO_INTERFACE_INVERSE) | \
            (0 if spectral else FP_NO_SPECTRAL)
        check(lib().fp_composite_create(ctypes.byref(g), int(m), float(tol), int(max_iter), flags, ctypes.byref(h)))
        self.h = h

    def set_parameter(self, m, tol, max_iter):
        check(lib().fp_composite_set_parameter(self.h, int(m), float(tol), int(max_iter)))

    def tree(self):
        root = ctypes.c_int(0)
        lv = np.zeros(self.nd, dtype=np.int32)
        check(lib().fp_composite_tree(self.h, ctypes.byref(root), lv.ctypes.data))
        return root.value, lv

    def _pointers(self, fields, ghosts):
        if len(fields) != self.nd:
            raise ValueError("one field per domain expected")
        keep, ptrs, flags, stream = [], [], 0, None
        for f, shp in zip(fields, self.shapes):
            if tuple(f.shape) != shp:
                raise ValueError(f"field shape {tuple(f.shape)} != domain shape {shp}")
            p, fl, st, k = _args(f, np.float64)
            if not _is_torch(f) and k is not f:
                raise TypeError("host fields must be contiguous float64 numpy arrays (solved in place)")
            flags |= fl
            stream = st if st is not None else stream
            keep.append(k)
            ptrs.append(p.value)
        fp = (ctypes.c_void_p * self.nd)(*ptrs)
        gp = None
        if ghosts is not None:
            gl = []
            for d in range(self.nd):
                for face in range(4):
                    gv = None if ghosts[d] is None else ghosts[d][face]
                    if gv is None:
                        gl.append(None)
                        continue
                    p, _, _, k = _args(gv, np.float64)
                    keep.append(k)
                    gl.append(p.value)
            gp = (ctypes.c_void_p * (4 * self.nd))(*gl)
        return fp, gp, flags, stream, keep

    @staticmethod
    def _info(info):
        return dict(iterations=info.gmres_iterations, restarts=info.gmres_restarts, residual=info.gmres_residual,
                    converged=bool(info.converged), refinements=info.refinements, rel_change=info.rel_change)

    def solve(self, fields, ghosts=None, check_convergence=False):
        """ConcatPoissonSolver2D::solve in place. fields: list of (nx, ny) float64 numpy arrays (host) or CUDA
        tensors (device). ghosts: None or per domain a list of 4 arrays/None (Variable2D buffer values)."""
        fp, gp, flags, stream, keep = self._pointers(fields, ghosts)
        info = SolveInfo()
        if check_convergence:
            flags |= FP_CHECK_CONVERGENCE
        check(lib().fp_composite_solve_f64(self.h, fp, gp, flags, stream, ctypes.byref(info)))
        return self._info(info)

    def solve_ir(self, fields, ghosts=None, rel_tol=1e-12, max_refine=10, check_convergence=False, inner="f32"):
        """The same solve by inner solves (FP32 transforms, FP64 with inner="f64", or inner="mixed": the FP64
        solve first, then FP32 corrections) wrapped in FP64 iterative refinement on the composite operator."""
        fp, gp, flags, stream, keep = self._pointers(fields, ghosts)
        info = SolveInfo()
        if check_convergence:
            flags |= FP_CHECK_CONVERGENCE
        if inner == "f64":
            flags |= FP_IR_INNER_F64
        elif inner == "mixed":
            flags |= FP_IR_FIRST_F64
        check(lib().fp_composite_solve_f32ir(self.h, fp, gp, flags, stream, float(rel_tol), int(max_refine),
                                             ctypes.byref(info)))
        return self._info(info)

    def _host_pointers(self, arrays, what):
        if len(arrays) != self.nd:
            raise ValueError(f"one {what} array per domain expected")
        ptrs = []
        for a, shp in zip(arrays, self.shapes):
            if tuple(a.shape) != shp:
                raise ValueError(f"{what} shape {tuple(a.shape)} != domain shape {shp}")
            if _is_torch(a):
                import torch

                if a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
                    raise TypeError(f"{what} tensors must be contiguous float64 host tensors")
                ptrs.append(a.data_ptr())
            else:
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                    raise TypeError(f"{what} arrays must be contiguous float64 numpy arrays")
                ptrs.append(a.ctypes.data)
        return ptrs

    def solve_async(self, rhs, out, ghosts=None, form="mixedir", rel_tol=1e-12, max_refine=10, stream=None):
        """Queue one solve of a stream of independent problems with host buffers (fp_composite_solve_async):
        rhs / out are per-domain host arrays (numpy or CPU torch tensors; page-locked memory lets the copies
        overlap the solves), out may be rhs. Returns at once; wait() finishes every queued call. The arrays are
        kept alive here until then and must not be touched meanwhile."""
        if form not in FORMS:
            raise ValueError(f"form must be one of {sorted(FORMS)}")
        rp = self._host_pointers(rhs, "rhs")
        op = self._host_pointers(out, "out")
        keep = [rhs, out, ghosts]
        gp = None
        if ghosts is not None:
            gl = []
            for d in range(self.nd):
                for face in range(4):
                    gv = None if ghosts[d] is None else ghosts[d][face]
                    if gv is None:
                        gl.append(None)
                        continue
                    if not (isinstance(gv, np.ndarray) and gv.dtype == np.float64 and gv.flags.c_contiguous):
                        raise TypeError("ghost buffers must be contiguous float64 numpy arrays")
                    gl.append(gv.ctypes.data)
            gp = (ctypes.c_void_p * (4 * self.nd))(*gl)
        st = None if stream is None else ctypes.c_void_p(int(stream))
        check(lib().fp_composite_solve_async(self.h, (ctypes.c_void_p * self.nd)(*rp),
                                             (ctypes.c_void_p * self.nd)(*op), gp, FORMS[form], float(rel_tol),
                                             int(max_refine), st))
        self.__dict__.setdefault("_queued", []).append(keep)

    def wait(self, check_convergence=False):
        """Wait for the solves queued by solve_async; returns the info of the last one."""
        info = SolveInfo()
        try:
            check(lib().fp_composite_wait(self.h, FP_CHECK_CONVERGENCE if check_convergence else 0,
                                          ctypes.byref(info)))
        finally:
            self.__dict__["_queued"] = []
        return self._info(info)

    def adjoint(self, fields, check_convergence=False):
        """Transposed solve in place: fields <- H A^-1 fields (the gradient with respect to the right-hand
        side of a loss whose gradient with respect to the solution is `fields`)."""
        fp, _, flags, stream, keep = self._pointers(fields, None)
        info = SolveInfo()
        if check_convergence:
            flags |= FP_CHECK_CONVERGENCE
        check(lib().fp_composite_adjoint_f64(self.h, fp, flags, stream, ctypes.byref(info)))
        return self._info(info)

    def adjoint_ir(self, fields, rel_tol=1e-12, max_refine=10, check_convergence=False, inner="f32"):
        """The transposed solve by iterative refinement (FP32 or FP64 inner solves, FP64 residual)."""
        fp, _, flags, stream, keep = self._pointers(fields, None)
        info = SolveInfo()
        if check_convergence:
            flags |= FP_CHECK_CONVERGENCE
        if inner == "f64":
            flags |= FP_IR_INNER_F64
        check(lib().fp_composite_adjoint_f32ir(self.h, fp, flags, stream, float(rel_tol), int(max_refine),
                                               ctypes.byref(info)))
        return self._info(info)

    def residual(self, u, rhs, ghosts=None):
        """|fs - A u| / |fs| for device tensors u (solution) and rhs (unassembled right-hand side)."""
        up, gp, _, stream, keep = self._pointers(u, ghosts)
        rp, _, _, _, keep2 = self._pointers(rhs, None)
        out = ctypes.c_double(0.0)
        check(lib().fp_composite_residual(self.h, up, rp, gp, stream, ctypes.byref(out)))
        return out.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_composite_destroy(self.h)
            self.h = None


class Batch:
    """Batched composite solves (fp_batch_*): `problems` is a list of geometries (as for Composite), each a
    root with leaves on full faces, Dirichlet outer faces, nx a multiple of 32. Fields are CUDA float64
    tensors, one per subdomain, problems back to back (flat list)."""

    def __init__(self, problems, precision="f64", autotune=True):
        self.keep = []
        geos = (Geometry * len(problems))()
        self.shapes = []
        for p, geo in enumerate(problems):
            arr = dict(
                nx=np.ascontiguousarray(geo.nx, dtype=np.int32), ny=np.ascontiguousarray(geo.ny, dtype=np.int32),
                hx=np.ascontiguousarray(geo.hx, dtype=np.float64), hy=np.ascontiguousarray(geo.hy, dtype=np.float64),
                bc=np.ascontiguousarray(np.asarray(geo.bc, dtype=np.int32).reshape(-1)),
                conn=np.ascontiguousarray(np.asarray(geo.connections, dtype=np.int32).reshape(-1)))
            self.keep.append(arr)
            nc = len(geo.connections)
            geos[p] = Geometry(len(geo.nx), arr["nx"].ctypes.data, arr["ny"].ctypes.data, arr["hx"].ctypes.data,
                               arr["hy"].ctypes.data, arr["bc"].ctypes.data, nc,
                               arr["conn"].ctypes.data if nc else None, -1)
            self.shapes += [(int(a), int(b)) for a, b in zip(geo.nx, geo.ny)]
        flags = (FP_BATCH_F32 if precision == "f32" else 0) | (0 if autotune else FP_BATCH_NO_AUTOTUNE)
        h = ctypes.c_void_p()
        check(lib().fp_batch_create(geos, len(problems), flags, ctypes.byref(h)))
        self.h = h
        self.n_problems = len(problems)
        self.n_domains = len(self.shapes)

    def _ptrs(self, fields):
        if len(fields) != self.n_domains:
            raise ValueError(f"{self.n_domains} fields expected")
        ptrs = []
        for f, shp in zip(fields, self.shapes):
            if tuple(f.shape) != shp:
                raise ValueError(f"field shape {tuple(f.shape)} != subdomain shape {shp}")
            p, fl, _, _ = _args(f, np.float64)
            if not fl & FP_DEVICE:
                raise TypeError("batched solves take CUDA tensors")
            ptrs.append(p.value)
        return (ctypes.c_void_p * self.n_domains)(*ptrs)

    def _ghosts(self, ghosts):
        if ghosts is None:
            return None
        gl = []
        for d in range(self.n_domains):
            for face in range(4):
                g = None if ghosts[d] is None else ghosts[d][face]
                gl.append(None if g is None else _args(g, np.float64)[0].value)
        return (ctypes.c_void_p * (4 * self.n_domains))(*gl)

    def solve(self, fields, ghosts=None, steps=0, graph=False, sync=False):
        """In place. steps == 0: one solve in the storage precision; steps >= 1: FP64 iterative refinement
        with that many inner solves. graph: capture once, replay afterwards (same tensors and steps)."""
        flags = FP_DEVICE | (FP_BATCH_GRAPH if graph else 0) | (FP_SYNC if sync else 0)
        check(lib().fp_batch_solve(self.h, self._ptrs(fields), self._ghosts(ghosts), flags, _stream(), int(steps)))

    def residuals(self, u, rhs, ghosts=None):
        out = np.zeros(self.n_problems)
        check(lib().fp_batch_residuals(self.h, self._ptrs(u), self._ptrs(rhs), self._ghosts(ghosts), _stream(),
                                       out.ctypes.data))
        return out

    def info(self):
        npb, nd, gk = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        shape = (ctypes.c_int * 3)()
        check(lib().fp_batch_info(self.h, ctypes.byref(npb), ctypes.byref(nd), shape, ctypes.byref(gk)))
        return dict(n_problems=npb.value, n_domains=nd.value, dst_threads=shape[0], dst_blocks_per_sm=shape[1],
                    chase_threads=shape[2], graph_kernels=gk.value)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fp_batch_destroy(self.h)
            self.h = None



# ---------------------------------------------------------------------------------------------------------
# Device-side field set-up (fp_field_fill / fp_buffer_fill)
# ---------------------------------------------------------------------------------------------------------
FACTOR_ONE, FACTOR_SIN, FACTOR_COS, FACTOR_GAUSS, FACTOR_QUADRATIC = range(5)
POS_CENTER, POS_XFACE, POS_YFACE, POS_CORNER = range(4)


class Term(ctypes.Structure):
    """a * X(x) * Y(y), factors FACTOR_* with parameters px, py (include/fp_capi.h fp_term)."""
    _fields_ = [("a", ctypes.c_double), ("kind_x", ctypes.c_int), ("kind_y", ctypes.c_int),
                ("px", ctypes.c_double * 3), ("py", ctypes.c_double * 3)]


def term(a, kx=FACTOR_ONE, px=(0.0, 0.0, 0.0), ky=FACTOR_ONE, py=(0.0, 0.0, 0.0)):
    px = tuple(px) + (0.0,) * (3 - len(px))
    py = tuple(py) + (0.0,) * (3 - len(py))
    return Term(float(a), int(kx), int(ky), (ctypes.c_double * 3)(*px), (ctypes.c_double * 3)(*py))


def _terms(terms):
    arr = (Term * max(1, len(terms)))(*terms)
    return arr, len(terms)


def field_fill(f, hx, hy, ox, oy, terms, position=POS_CENTER, accumulate=False):
    """Variable2D::set_value on the device: f (an (nx, ny) CUDA float64 tensor) = the sum of `terms` at the
    value positions of a domain with offset (ox, oy) and steps hx, hy."""
    import torch

    nx, ny = f.shape
    arr, n = _terms(terms)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().fp_field_fill(ctypes.c_void_p(f.data_ptr()), nx, ny, float(hx), float(hy), float(ox), float(oy),
                              int(position), arr, n, int(bool(accumulate)), s))
    return f


def buffer_fill(buf, face, nx, ny, hx, hy, ox, oy, terms, position=POS_CENTER):
    """Variable2D::set_buffer_value on the device: the ghost values of `face` into the CUDA tensor buf."""
    import torch

    arr, n = _terms(terms)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().fp_buffer_fill(ctypes.c_void_p(buf.data_ptr()), int(face), nx, ny, float(hx), float(hy), float(ox),
                               float(oy), int(position), arr, n, s))
    return buf
