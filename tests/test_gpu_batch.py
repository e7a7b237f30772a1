"""GPU parity of the batched composite solves (fp_batch_*): small L/T problems and 64^2 crosses with Neumann
arm tips and ghost values against the reference's own converged solutions (tests/golden/batch_lt_*.npz,
cross64_*.npz), larger ones against the single-problem C-ABI Schur GMRES solve,
graph capture/replay, per-problem residuals, the unsupported cases, and the full batched-uneven workload
(512 L/T problems, sides 64..1024) checked through residuals and sampled problems."""
import types

import numpy as np
import pytest

from golden_io import composite_case, rel_l2, tight_outputs
from gpu_util import torch_cuda
from focalors_poisson_b200 import capi
from focalors_poisson_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = [f"batch_lt_{k}.npz" for k in range(4)] + ["cross64_neumann_tips.npz", "cross64_ghosts.npz"]


def _golden_problems():
    probs, rhs, ghosts, tight = [], [], [], []
    for name in GOLDEN:
        geo, r, gh, _, _, _ = composite_case(name)
        probs.append(types.SimpleNamespace(**geo))
        rhs += list(r)
        ghosts += gh if gh is not None else [None] * len(r)
        tight += tight_outputs(name)
    return probs, rhs, ghosts, tight


def _split(fields, probs):
    out, k = [], 0
    for g in probs:
        out.append(fields[k:k + len(g.nx)])
        k += len(g.nx)
    return out


@pytest.mark.parametrize("precision,steps,tol", [("f64", 0, 1e-11), ("f64", 2, 1e-12), ("f32", 0, 1e-4),
                                                 ("f32", 2, 1e-10), ("f32", 3, 1e-10)])
def test_batch_against_reference(precision, steps, tol):
    torch = torch_cuda()
    probs, rhs, ghosts, tight = _golden_problems()
    b = capi.Batch(probs, precision=precision)
    f = [torch.tensor(r, device="cuda") for r in rhs]
    gh = [None if g is None else [None if x is None else torch.tensor(x, device="cuda") for x in g] for g in ghosts]
    b.solve(f, gh, steps=steps)
    torch.cuda.synchronize()
    got = [x.cpu().numpy() for x in f]
    for p, (a, t) in enumerate(zip(_split(got, probs), _split(tight, probs))):
        assert rel_l2(a, t) <= tol, (p, rel_l2(a, t))


def test_batch_matches_single_problem_solves():
    torch = torch_cuda()
    probs = [W.lt_problem(100 + p, sides=W.SIDES[:12]) for p in range(6)]
    rhs = [x for p, g in enumerate(probs) for x in W.gaussian_rhs(g, 900 + p, zero_mean=False)]
    b = capi.Batch(probs)
    f = [torch.tensor(r, device="cuda") for r in rhs]
    b.solve(f, steps=1)
    torch.cuda.synchronize()
    for p, (g, got) in enumerate(zip(probs, _split([x.cpu().numpy() for x in f], probs))):
        want = [np.array(r, copy=True) for r in _split(rhs, probs)[p]]
        capi.Composite(g, 20, 1e-14, 200, spectral=False).solve(want)
        assert rel_l2(got, want) <= 1e-11, (p, rel_l2(got, want))


def test_batch_graph_replay_and_residuals():
    torch = torch_cuda()
    probs, rhs, _, tight = _golden_problems()
    b = capi.Batch(probs, precision="f32")
    pristine = [torch.tensor(r, device="cuda") for r in rhs]
    plain = [x.clone() for x in pristine]
    b.solve(plain, steps=3)
    f = [x.clone() for x in pristine]
    for _ in range(3):  # replays of one captured graph on the same tensors
        for x, p in zip(f, pristine):
            x.copy_(p)
        b.solve(f, steps=3, graph=True)
    torch.cuda.synchronize()
    assert b.info()["graph_kernels"] > 0
    for x, y in zip(f, plain):
        assert torch.equal(x, y)
    res = b.residuals(f, pristine)
    assert res.shape == (len(probs),) and float(res.max()) <= 1e-11, res


def test_batch_rejects_unsupported():
    torch_cuda()
    g = W.lt_problem(1, sides=(64,))
    bad = types.SimpleNamespace(**{k: getattr(g, k) for k in ("nx", "ny", "hx", "hy", "connections")})
    bad.bc = [list(r) for r in g.bc]
    bad.bc[0][W.YNEG] = W.NEUMANN  # Neumann on the root
    with pytest.raises(capi.FpError) as e:
        capi.Batch([bad])
    assert e.value.code == 3
    side = types.SimpleNamespace(**{k: getattr(g, k) for k in ("nx", "ny", "hx", "hy", "connections")})
    side.bc = [list(r) for r in g.bc]
    side.bc[1][W.YNEG] = W.NEUMANN  # Neumann on an x-leaf's side along the interface
    with pytest.raises(capi.FpError) as e:
        capi.Batch([side])
    assert e.value.code == 3
    odd = types.SimpleNamespace(nx=[48, 48], ny=[32, 32], hx=[0.1, 0.1], hy=[0.1, 0.1], bc=[[0] * 4] * 2,
                                connections=[(0, W.XPOS, 1)])
    with pytest.raises(capi.FpError) as e:
        capi.Batch([odd])
    assert e.value.code == 3


def test_batched_uneven_workload_512():
    """The full workload: 512 problems, FP32 storage + FP64 refinement (2 and 3 inner solves; the first
    one's inverse transform in FP64 arithmetic) in one captured graph, and the FP64 direct solve; every
    problem's residual small, four sampled problems equal to the single-problem C-ABI solve."""
    torch = torch_cuda()
    probs, rhs = W.batched_uneven(512)
    flat = [x for r in rhs for x in r]
    pristine = [torch.tensor(x, device="cuda") for x in flat]
    # residual bounds: FP64 direct 1e-11 (the solve's round-off floor at 1024^2), FP32 with 3 inner solves
    # 5e-9, with 2 inner solves 2e-8: the last FP32 correction's storage rounding leaves a rough error of
    # ~1e-14, and a rough error's residual at 1024^2 is up to ~8 / lambda_min ~ 4e5 times larger; the error
    # itself is checked against the single-problem solves below
    for precision, steps, rtol, etol in (("f32", 2, 2e-8, 1e-10), ("f32", 3, 5e-9, 1e-10),
                                         ("f64", 0, 5e-11, 1e-10)):
        b = capi.Batch(probs, precision=precision)
        f = [x.clone() for x in pristine]
        b.solve(f, steps=steps, graph=True)
        torch.cuda.synchronize()
        res = b.residuals(f, pristine)
        assert float(res.max()) <= rtol, (precision, float(res.max()))
        k = 0
        starts = np.cumsum([0] + [len(g.nx) for g in probs])
        for p in (0, 17, 255, 511):
            want = [np.array(x, copy=True) for x in rhs[p]]
            capi.Composite(probs[p], 20, 1e-14, 200, spectral=False).solve(want)
            got = [f[starts[p] + d].cpu().numpy() for d in range(len(probs[p].nx))]
            assert rel_l2(got, want) <= etol, (precision, p, rel_l2(got, want))
        del b, f
        torch.cuda.empty_cache()
