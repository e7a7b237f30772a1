"""fp_rect_solve_f64_noalloc: the rectangle solve for callers that cannot allocate device memory when
they solve (their device memory belongs to another allocator or a fixed budget). Its scratch is one fixed
device array shared by every call; this checks it against the allocating entry point, fp_rect_solve_f64,
on two calls in a row (the array keeps the previous call's contents), and that oversize solves are
refused. Kept in a file pytest collects last."""
import ctypes

import numpy as np
import pytest

from focalors_poisson_b200 import capi

pytestmark = pytest.mark.gpu


def _solve_noalloc(rect, t, torch):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    batch = t.shape[0] if t.dim() == 3 else 1
    return capi.lib().fp_rect_solve_f64_noalloc(rect.h, ctypes.c_void_p(t.data_ptr()), batch, stream)


@pytest.mark.parametrize("shape,bc", [((128, 96, 1 / 128, 1 / 96), (0, 1, 1, 0)),
                                      ((64, 40, 0.1, 0.2), (1, 1, 1, 1)),
                                      ((96, 50, 0.02, 0.02), (1, 0, 2, 2))])
def test_noalloc_matches_allocating_entry_point(shape, bc):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    nx, ny, hx, hy = shape
    rect = capi.Rect(nx, ny, hx, hy, bc)
    rng = np.random.default_rng(nx * ny)
    for _ in range(2):
        f = rng.standard_normal((3, nx, ny))
        want = torch.tensor(f, device="cuda")
        got = want.clone()
        rect.solve(want)
        assert _solve_noalloc(rect, got, torch) == 0, capi.lib().fp_last_error()
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), want.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_noalloc_refuses_oversize_batch():
    torch = pytest.importorskip("torch")
    n = 2048
    rect = capi.Rect(n, n, 1 / n, 1 / n, (0, 0, 0, 0))
    # 4 * batch * (n/32) * n doubles: batch 5 needs 2,621,440 > 2^21
    t = torch.zeros((5, n, n), dtype=torch.float64, device="cuda")
    rc = _solve_noalloc(rect, t, torch)
    assert rc == 3  # FP_ERR_UNSUPPORTED
    assert "no-allocation scratch" in capi.lib().fp_last_error().decode()
    assert _solve_noalloc(rect, t[:4], torch) == 0
