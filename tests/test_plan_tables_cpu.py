"""CPU check of the host-side Bluestein plans (no GPU): the driver tests/cases/plan_tables.cu prints a
plan's window, length M, stage radices, chirp and kernel transforms; numpy replays the algorithm the device
engine runs on those tables (pre-chirp on the input window, cyclic convolution of length M through the
digit-reversed kernel transform, post-chirp on the output window) and compares it with a direct DFT of
length L. This pins the choice of M (2L-2 for the full window, nin + nout - 1 for the quarter-wave
windows) and the tables independently of the device butterflies, which the GPU tests cover."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cases", "plan_tables.cu")
PLAN = os.path.join(ROOT, "focalors_poisson_b200", "csrc", "fp_plan.cu")
K_DD, K_NN, K_ND, K_DN = 0, 1, 2, 3


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("plan") / "plan_tables")
    subprocess.run([nvcc, "-std=c++17", "-O1", SRC, PLAN, "-o", out], check=True, capture_output=True)
    return out


def plan(driver, kind, n):
    txt = subprocess.run([driver, str(kind), str(n)], check=True, capture_output=True, text=True).stdout
    p = {"c": [], "b": [], "i": []}
    for line in txt.splitlines():
        f = line.split()
        if f[0] in ("fwd", "inv"):
            p[f[0]] = dict(zip(("L", "M", "blue", "in0", "nin", "out0", "nout"), map(int, f[1:])))
        elif f[0] == "radices":
            p["radices"] = [int(x) for x in f[1:]]
        else:
            p[f[0]].append(complex(float(f[1]), float(f[2])))
    for k in ("c", "b", "i"):
        p[k] = np.array(p[k])
    return p


def dif_frequency(M, radices):
    """Frequency held by slot p after the DIF stages (the plan's digit-reversed order)."""
    k = np.zeros(M, dtype=np.int64)
    for p in range(M):
        pp, mult, S, kk = p, 1, M, 0
        for r in radices:
            S //= r
            d = pp // S
            pp -= d * S
            kk += d * mult
            mult *= r
        k[p] = kk
    return k


def replay(p, w, bhat, z):
    """Bluestein on the plan's tables: X_{out0+t} for t < nout from input z (length L)."""
    M = p["fwd"]["M"]
    c = p["c"]
    a = np.zeros(M, complex)
    a[: w["nin"]] = z[w["in0"]: w["in0"] + w["nin"]] * c[w["in0"]: w["in0"] + w["nin"]]
    kern = np.zeros(M, complex)
    kern[dif_frequency(M, p["radices"])] = bhat * M  # natural order, unscaled
    y = np.fft.ifft(np.fft.fft(a) * kern)
    t = np.arange(w["nout"])
    return c[w["out0"] + t] * y[: w["nout"]]


@pytest.mark.parametrize("kind,n", [(K_DD, 2048), (K_DD, 1000), (K_DD, 96), (K_ND, 2048), (K_ND, 130),
                                    (K_DN, 1000), (K_DN, 64), (K_NN, 352)])
def test_bluestein_tables_replay_dft(driver, kind, n):
    p = plan(driver, kind, n)
    f = p["fwd"]
    assert f["blue"] == 1
    L, M = f["L"], f["M"]
    full = f["nin"] == L and f["nout"] == L
    need = 2 * L - 2 if full else max(f["nin"] + f["nout"], p["inv"]["nin"] + p["inv"]["nout"]) - 1
    assert M >= need and M <= need + need // 2
    if kind in (K_ND, K_DN):
        assert (f["in0"], f["nin"], f["out0"], f["nout"]) == (1, n, 1, 2 * n)
    if kind == K_DD and n == 2048:
        assert M == 4096  # 2L - 2: a power of two instead of 4116 = 4 * 3 * 7^3
    if kind == K_ND and n == 2048:
        assert M == 6144  # 3n - 1 rounded up to a smooth length, instead of 8192
    rng = np.random.default_rng(n + kind)
    for tag, bhat in (("fwd", p["b"]), ("inv", p["i"] if len(p["i"]) else p["b"])):
        w = p[tag]
        z = np.zeros(L, complex)
        z[w["in0"]: w["in0"] + w["nin"]] = rng.standard_normal(w["nin"]) + 1j * rng.standard_normal(w["nin"])
        ref = np.fft.fft(z)[w["out0"]: w["out0"] + w["nout"]]
        got = replay(p, w, bhat, z)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (kind, n, tag)
    if kind == K_ND:
        assert len(p["i"]) == M  # the inverse window has its own kernel table
        assert (p["inv"]["in0"], p["inv"]["nin"], p["inv"]["out0"], p["inv"]["nout"]) == (1, 2 * n, 1, n)


@pytest.mark.parametrize("kind", [K_DD, K_ND, K_DN])
def test_bluestein_tables_batch_sizes(driver, kind):
    """Row lengths of the batched workload (multiples of 32 in 64..1024): every Bluestein plan replays the DFT
    on both windows, and its length is the cheapest smooth one at or above what the window needs."""
    rng = np.random.default_rng(kind)
    checked = 0
    for n in range(64, 1025, 96):
        p = plan(driver, kind, n)
        f = p["fwd"]
        if not f["blue"]:
            continue
        L, M = f["L"], f["M"]
        full = f["nin"] == L and f["nout"] == L
        need = 2 * L - 2 if full else max(f["nin"] + f["nout"], p["inv"]["nin"] + p["inv"]["nout"]) - 1
        assert need <= M <= need + need // 2, (kind, n, M)
        for tag, bhat in (("fwd", p["b"]), ("inv", p["i"] if len(p["i"]) else p["b"])):
            w = p[tag]
            z = np.zeros(L, complex)
            z[w["in0"]: w["in0"] + w["nin"]] = rng.standard_normal(w["nin"]) + 1j * rng.standard_normal(w["nin"])
            ref = np.fft.fft(z)[w["out0"]: w["out0"] + w["nout"]]
            got = replay(p, w, bhat, z)
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (kind, n, tag)
        checked += 1
    assert checked >= 5
