"""GPU parity of the 3D composite solve (ConcatPoissonSolver3D) against the reference's own outputs
(tests/golden/concat3d.npz, generated from its sources) through the C ABI."""
import numpy as np
import pytest

from golden_io import CONCAT3D_CASES, concat3d_case, rel_l2
from gpu_util import torch_cuda
from focalors_poisson_b200 import capi

pytestmark = pytest.mark.gpu


def _solver(name, tol=1e-12):
    doms, conns, bc, rhs, ghosts, outs, tight, root, levels = concat3d_case(name)
    return capi.Composite3D(doms, conns, bc, 20, tol, 100), rhs, ghosts, outs, tight, root, levels


@pytest.mark.parametrize("name", CONCAT3D_CASES)
def test_concat3d_matches_reference(name):
    """Same tree as the reference; the solve at the case's GMRES tolerance matches the reference's solve at the
    same tolerance, and the solve at 1e-15 matches the reference's at 1e-15."""
    solver, rhs, ghosts, outs, tight, root, levels = _solver(name)
    r, lv = solver.tree()
    assert r == root and (lv == levels).all()
    f = [np.array(x, dtype=np.float64, copy=True) for x in rhs]
    info = solver.solve(f, ghosts)
    assert info["converged"]
    assert rel_l2(f, outs) <= 1e-10, name
    solver.set_parameter(20, 1e-15, 100)
    f = [np.array(x, dtype=np.float64, copy=True) for x in rhs]
    solver.solve(f, ghosts)
    assert rel_l2(f, tight) <= 1e-12, name


def test_concat3d_device_fields():
    """Device tensors (FP_DEVICE) give the host path's answer."""
    torch = torch_cuda()
    solver, rhs, ghosts, outs, tight, root, levels = _solver("star")
    host = [np.array(x, dtype=np.float64, copy=True) for x in rhs]
    solver.solve(host, ghosts)
    dev = [torch.tensor(x, device="cuda") for x in rhs]
    gdev = [[torch.tensor(g, device="cuda") for g in gs] for gs in ghosts]
    solver.solve(dev, gdev)
    torch.cuda.synchronize()
    assert rel_l2([d.cpu().numpy() for d in dev], host) <= 1e-14


def test_concat3d_geometry_errors():
    with pytest.raises(capi.FpError):  # connected faces of different sizes
        capi.Composite3D([(8, 8, 8, 0.1, 0.1, 0.1), (8, 6, 8, 0.1, 0.1, 0.1)], [(0, 1, 1)], [[0] * 6] * 2)
    with pytest.raises(capi.FpError):  # a cycle
        capi.Composite3D([(4, 4, 4, 0.1, 0.1, 0.1)] * 3, [(0, 1, 1), (1, 1, 2), (2, 1, 0)], [[0] * 6] * 3)
