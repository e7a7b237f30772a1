"""Device-side field set-up (fp_field_fill / fp_buffer_fill) against the values Variable2D::set_value and
set_buffer_value compute on the host (reference base/domain/variable2d.cpp:345-416, 467-511): the same
function at the same positions, evaluated here in numpy."""
import numpy as np
import pytest

from gpu_util import torch_cuda
from focalors_poisson_b200 import capi

pytestmark = pytest.mark.gpu

TERMS = [capi.term(1.3, capi.FACTOR_SIN, (np.pi, 0.0), capi.FACTOR_SIN, (np.pi, 0.2)),
         capi.term(-0.7, capi.FACTOR_GAUSS, (1.4, 0.05), capi.FACTOR_GAUSS, (0.6, 0.03)),
         capi.term(0.25, capi.FACTOR_QUADRATIC, (1.0, -2.0, 0.5), capi.FACTOR_COS, (3.0, 1.0)),
         capi.term(2.0)]


def f_np(x, y):
    return (1.3 * np.sin(np.pi * x) * np.sin(np.pi * y + 0.2) - 0.7 * np.exp(-((x - 1.4) / 0.05) ** 2) *
            np.exp(-((y - 0.6) / 0.03) ** 2) + 0.25 * (1.0 - 2.0 * x + 0.5 * x * x) * np.cos(3.0 * y + 1.0) + 2.0)


SHIFT = {capi.POS_CENTER: (0.5, 0.5), capi.POS_XFACE: (0.0, 0.5), capi.POS_YFACE: (0.5, 0.0), capi.POS_CORNER: (0.0, 0.0)}


@pytest.mark.parametrize("position", list(SHIFT))
def test_field_fill_matches_set_value_positions(position):
    torch = torch_cuda()
    nx, ny, hx, hy, ox, oy = 96, 80, 1 / 64, 1 / 48, 1.0, 0.5
    f = torch.zeros((nx, ny), dtype=torch.float64, device="cuda")
    capi.field_fill(f, hx, hy, ox, oy, TERMS, position)
    sx, sy = SHIFT[position]
    x = ox + (np.arange(nx)[:, None] + sx) * hx
    y = oy + (np.arange(ny)[None, :] + sy) * hy
    want = f_np(x, y)
    got = f.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
    capi.field_fill(f, hx, hy, ox, oy, TERMS[:1], position, accumulate=True)  # += one term
    want2 = want + 1.3 * np.sin(np.pi * x) * np.sin(np.pi * y + 0.2)
    assert np.abs(f.cpu().numpy() - want2).max() <= 1e-14 * np.abs(want2).max()


@pytest.mark.parametrize("position", [capi.POS_CENTER, capi.POS_CORNER])
def test_buffer_fill_matches_set_buffer_value_positions(position):
    torch = torch_cuda()
    nx, ny, hx, hy, ox, oy = 40, 24, 0.05, 0.04, -0.3, 0.2
    sx, sy = SHIFT[position]
    extra = 1 if position == capi.POS_CORNER else 0
    for face in range(4):
        n = (ny if face < 2 else nx) + extra
        b = torch.zeros(n, dtype=torch.float64, device="cuda")
        capi.buffer_fill(b, face, nx, ny, hx, hy, ox, oy, TERMS, position)
        k = np.arange(n)
        if face < 2:  # ghost column one cell outside the x face (variable2d.cpp:386-394)
            x = ox + (sx + (-1 if face == 0 else nx)) * hx + 0 * k
            y = oy + (sy + k) * hy
        else:
            x = ox + (sx + k) * hx
            y = oy + (sy + (-1 if face == 2 else ny)) * hy + 0 * k
        want = f_np(x, y)
        assert np.abs(b.cpu().numpy() - want).max() <= 1e-14 * np.abs(want).max(), face


def test_field_fill_rejects_bad_arguments():
    torch = torch_cuda()
    f = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.FpError) as e:
        capi.field_fill(f, 0.1, 0.1, 0, 0, [capi.term(1.0)] * 49)
    assert e.value.code == 3
    with pytest.raises(capi.FpError):
        capi.field_fill(f, 0.1, 0.1, 0, 0, [capi.term(1.0, capi.FACTOR_GAUSS, (0.0, 0.0))])
