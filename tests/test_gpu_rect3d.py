"""GPU parity of the 3D rectangle solve (PoissonSolver3D, fp_rect3d_*) against the reference's own output
(tests/golden/poisson3d.npz, generated from its sources) and, at larger sizes, against the reference library
itself (oracle/_ref), through the C ABI."""
import numpy as np
import pytest

from golden_io import load
from gpu_util import rel_max, torch_cuda
from focalors_poisson_b200 import capi
from oracle import refbind as R

pytestmark = pytest.mark.gpu


def test_rect3d_golden_all_boundary_combinations():
    z = load("poisson3d.npz")
    f = z["small_in"]
    for c, bc in enumerate(z["combos"]):
        got = capi.Rect3D(6, 6, 4, 0.3, 0.2, 0.25, [int(b) for b in bc]).solve(f.copy())
        assert rel_max(got, z[f"small_{c}"]) <= 1e-12, (c, bc)
    for tag in ("a", "b"):  # 64 cells along x: the partition chase over the combined (z, y) modes
        g = z[f"{tag}_in"]
        got = capi.Rect3D(*g.shape, *z[f"{tag}_h"], [int(b) for b in z[f"{tag}_bc"]]).solve(g.copy())
        assert rel_max(got, z[f"{tag}_out"]) <= 1e-12, tag


@pytest.mark.parametrize("shape,bc", [((128, 96, 64), (0, 0, 0, 0, 0, 0)), ((96, 64, 80), (1, 0, 0, 1, 2, 2)),
                                      ((50, 40, 48), (2, 2, 1, 1, 1, 1)), ((64, 48, 32), (1, 1, 1, 1, 1, 1))])
def test_rect3d_matches_reference_library(shape, bc):
    """Larger fields through device pointers, two fields in one call, against the reference's PoissonSolver3D
    (oracle/_ref). The third case has no Dirichlet face and periodic x, where the reference treats every
    y-mode of the last z-mode as singular; the fourth has no Dirichlet face and the partition chase."""
    torch = torch_cuda()
    assert R.available(), "oracle/_ref/libfpref.so (the reference's own sources, built by build()) is missing"
    nx, ny, nz = shape
    h = (1.0 / nx, 1.0 / ny, 1.0 / nz)
    rng = np.random.default_rng(nx + ny + nz)
    f = rng.standard_normal((2, nx, ny, nz))
    t = torch.tensor(f, device="cuda")
    capi.Rect3D(nx, ny, nz, *h, bc).solve(t)
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    for b in range(2):
        want = R.poisson3d_solve(f[b], *h, bc)[0]
        assert rel_max(got[b], want) <= 1e-11, (shape, bc, b)
