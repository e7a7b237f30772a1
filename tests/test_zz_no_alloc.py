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


# the first three take the partition chase (nx a multiple of 32, x not periodic), which uses the fixed
# scratch; the last two the sequential chase (nx = 50; periodic x), which needs none
@pytest.mark.parametrize("shape,bc", [((128, 96, 1 / 128, 1 / 96), (0, 1, 1, 0)),
                                      ((64, 40, 0.1, 0.2), (1, 1, 1, 1)),
                                      ((96, 50, 0.02, 0.02), (1, 0, 2, 2)),
                                      ((50, 40, 0.1, 0.1), (0, 1, 1, 0)),
                                      ((64, 48, 0.05, 0.05), (2, 2, 0, 1))])
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


def test_noalloc_allocates_no_device_memory():
    """The defining property: a solve that needs the full 16 MiB of scratch (2048^2, batch 4) takes no
    device memory of its own. The fixed array is loaded with the library's code, so one earlier call is
    made first; then a fresh solver's first no-allocation call must leave the device's free memory as it
    was (the allocating entry point would grow that solver's scratch by 16 MiB here)."""
    torch = pytest.importorskip("torch")
    n = 2048
    warm = capi.Rect(64, 64, 1 / 64, 1 / 64, (0, 0, 0, 0))
    t = torch.zeros((1, 64, 64), dtype=torch.float64, device="cuda")
    assert _solve_noalloc(warm, t, torch) == 0
    rect = capi.Rect(n, n, 1 / n, 1 / n, (0, 0, 0, 0))
    f = torch.randn((4, n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert _solve_noalloc(rect, f, torch) == 0, capi.lib().fp_last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < 16 * 2 ** 20, (free0, free1)
