"""GPU parity of the y-transforms and the single-rectangle solver against the reference (golden vectors
from its own sources) and the oracle, through the C ABI."""
import numpy as np
import pytest

from golden_io import load
from gpu_util import rel_max, torch_cuda
from oracle import fp_oracle as O
from focalors_poisson_b200 import capi

pytestmark = pytest.mark.gpu
PAIRS = {"DD": (0, 0), "NN": (1, 1), "ND": (1, 0), "DN": (0, 1), "PP": (2, 2)}


def test_transforms_golden_f64_host_and_device():
    torch = torch_cuda()
    z = load("transforms.npz")
    n = 0
    for key in z.files:
        if not key.startswith("in_"):
            continue
        _, kind, ny = key.split("_")
        f = z[key]
        for inv, tag in ((False, "fwd"), (True, "inv")):
            ref = z[f"{tag}_{kind}_{ny}"]
            got = capi.transform(*PAIRS[kind], f, inverse=inv)
            assert rel_max(got, ref) <= 1e-13, (kind, ny, tag)
            t = torch.tensor(f, device="cuda")
            got_d = capi.transform(*PAIRS[kind], t, inverse=inv).cpu().numpy()
            assert rel_max(got_d, ref) <= 1e-13, (kind, ny, tag, "device")
            n += 1
    assert n >= 100


@pytest.mark.parametrize("kind", list(PAIRS))
@pytest.mark.parametrize("ny", [6, 64, 130, 256, 1000, 2048, 3000, 4096])
def test_transforms_large_vs_oracle(kind, ny):
    rng = np.random.default_rng(ny)
    f = rng.standard_normal((5, ny))
    for inv in (False, True):
        ref = (O.transform_inverse if inv else O.transform_forward)(kind, f)
        got = capi.transform(*PAIRS[kind], f, inverse=inv)
        assert rel_max(got, ref) <= 1e-13, (kind, ny, inv)
        got32 = capi.transform(*PAIRS[kind], f.astype(np.float32), inverse=inv)
        assert rel_max(got32, ref) <= 2e-5, (kind, ny, inv, "f32")


@pytest.mark.parametrize("kind", list(PAIRS))
@pytest.mark.parametrize("ny", [7002, 12000, 20000])
def test_transforms_long_rows_vs_oracle(kind, ny):
    """Rows whose FFT buffer does not fit in a CTA's shared memory (FP64 ND/DN beyond ~4260, DD beyond ~6400;
    FP32 at twice those) run with the buffer in global memory: same results as the oracle."""
    rng = np.random.default_rng(ny + 7)
    f = rng.standard_normal((3, ny))
    for inv in (False, True):
        ref = (O.transform_inverse if inv else O.transform_forward)(kind, f)
        got = capi.transform(*PAIRS[kind], f, inverse=inv)
        assert rel_max(got, ref) <= 1e-12, (kind, ny, inv)
        got32 = capi.transform(*PAIRS[kind], f.astype(np.float32), inverse=inv)
        assert rel_max(got32, ref) <= 1e-4, (kind, ny, inv, "f32")


@pytest.mark.parametrize("bc", [(0, 0, 0, 0), (1, 0, 1, 0), (0, 1, 0, 1), (1, 1, 1, 1), (0, 0, 2, 2)])
def test_rect_long_rows_vs_oracle(bc):
    """PoissonSolver2D with ny = 9000 (beyond the shared-memory plans of every family): FP64 solve equals the
    oracle's."""
    torch = torch_cuda()
    nx, ny = 64, 9000
    rng = np.random.default_rng(5)
    f = rng.standard_normal((2, nx, ny))
    ref = np.stack([O.PoissonSolver2D(nx, ny, 1.0 / nx, 1.0 / ny, bc).solve(f[b]) for b in range(2)])
    t = torch.tensor(f, device="cuda")
    capi.Rect(nx, ny, 1.0 / nx, 1.0 / ny, bc).solve(t)
    assert rel_max(t.cpu().numpy(), ref) <= 1e-10, bc


def test_poisson_reference_driver_fixture():
    """case/validation/2d/poisson_solver_reference.cpp: 3x4, hx=1, hy=2, all 25 boundary combinations."""
    z = load("poisson.npz")
    f0 = np.arange(12, dtype=np.float64).reshape(3, 4) + 1.0
    for c, bc in enumerate(z["combos"]):
        f = f0.copy()
        capi.Rect(3, 4, 1.0, 2.0, bc).solve(f)
        assert rel_max(f, z[f"fixture_{c}"]) <= 1e-12, (c, bc)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_poisson_random_golden(tag):
    z = load("poisson.npz")
    f0 = z[f"rand_{tag}_in"]
    nx, ny, hx, hy = z[f"rand_{tag}_shape"]
    for c, bc in enumerate(z["combos"]):
        key = f"rand_{tag}_{c}"
        if key not in z.files:
            continue
        f = f0.copy()
        capi.Rect(int(nx), int(ny), hx, hy, bc).solve(f)
        assert rel_max(f, z[key]) <= 1e-11, (tag, c, bc)


@pytest.mark.parametrize("shape", [(64, 130, 1 / 64, 1 / 130), (128, 128, 1 / 128, 1 / 128), (40, 512, 0.01, 0.002)])
def test_rect_batched_device_vs_oracle(shape):
    torch = torch_cuda()
    nx, ny, hx, hy = shape
    rng = np.random.default_rng(nx + ny)
    combos = [(0, 0, 0, 0), (1, 0, 0, 1), (0, 1, 1, 0), (1, 1, 0, 0), (0, 0, 1, 1), (1, 1, 1, 1), (2, 2, 0, 1),
              (0, 1, 2, 2), (2, 2, 2, 2)]
    for bc in combos:
        f = rng.standard_normal((3, nx, ny))
        ref = np.stack([O.PoissonSolver2D(nx, ny, hx, hy, bc).solve(f[b]) for b in range(3)])
        t = torch.tensor(f, device="cuda")
        capi.Rect(nx, ny, hx, hy, bc).solve(t)
        assert rel_max(t.cpu().numpy(), ref) <= 1e-11, bc
        t32 = torch.tensor(f, device="cuda", dtype=torch.float32)
        capi.Rect(nx, ny, hx, hy, bc, precision=capi.FP_F32).solve(t32)
        assert rel_max(t32.double().cpu().numpy(), ref) <= 5e-3, (bc, "f32")


@pytest.mark.parametrize("nx,ny,bc", [(128, 96, (0, 1, 1, 0)), (50, 64, (1, 1, 0, 0)), (64, 40, (2, 2, 1, 1))])
def test_chase_entry_composes_the_solve(nx, ny, bc):
    """fp_rect_chase_f64 is the solve's middle step: forward transform, chase, inverse transform through three
    separate C-ABI calls equal one fp_rect_solve_f64."""
    torch = torch_cuda()
    rect = capi.Rect(nx, ny, 1.0 / nx, 1.0 / ny, bc)
    f = torch.randn(2, nx, ny, dtype=torch.float64, device="cuda")
    want = f.clone()
    rect.solve(want)
    got = f.clone()
    capi.transform(bc[2], bc[3], got, out=got)
    rect.chase(got)
    capi.transform(bc[2], bc[3], got, inverse=True, out=got)
    torch.cuda.synchronize()
    assert rel_max(got.cpu().numpy(), want.cpu().numpy()) <= 1e-13
