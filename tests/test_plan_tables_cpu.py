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


def plan(driver, kind, n, engine="stage"):
    txt = subprocess.run([driver, str(kind), str(n), engine], check=True, capture_output=True, text=True).stdout
    p = {"c": [], "b": [], "i": [], "t": []}
    for line in txt.splitlines():
        f = line.split()
        if f[0] in ("fwd", "inv"):
            p[f[0]] = dict(zip(("L", "M", "blue", "in0", "nin", "out0", "nout", "eng", "lgM"), map(int, f[1:])))
        elif f[0] == "radices":
            p["radices"] = [int(x) for x in f[1:]]
        else:
            p[f[0]].append(complex(float(f[1]), float(f[2])))
    for k in ("c", "b", "i", "t"):
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


# ---------------------------------------------------------------------------------------------------
# Register engine (csrc/fp_fft16.cuh): Stockham passes on 16 registers per thread, replayed in numpy with
# the plan's own tables
# ---------------------------------------------------------------------------------------------------
def reg_fft(x, tw):
    """The register engine's forward FFT of x (length M = 2^m >= 512) with its pass order (a radix
    2^(m mod 4) pass first, then radix-16 passes), the column layout of thread t (elements t + T q), the
    exchange destinations (j / Ns) Ns R + j mod Ns + r Ns and the rotation base tw[(j mod Ns) M / (16 Ns)]."""
    M = len(x)
    T = M // 16
    m = M.bit_length() - 1
    radices = ([2 ** (m % 4)] if m % 4 else []) + [16] * (m // 4)
    col = x.reshape(16, T).T.copy()  # col[t, q] = x[t + T q]
    Ns = 1
    for R in radices:
        B = 16 // R
        dest = np.zeros(M, complex)
        last = Ns * R == M
        for t in range(T):
            for b in range(B):
                j = t + b * T
                q = b + np.arange(R) * B
                legs = col[t, q]
                k = j % Ns
                if Ns > 1 and k:
                    legs = legs * tw[k * (M // (16 * Ns))] ** np.arange(R)
                out = np.fft.fft(legs)
                if last:
                    col[t, q] = out
                else:
                    dest[(j // Ns) * Ns * R + k + np.arange(R) * Ns] = out
        if not last:
            col = dest.reshape(16, T).T.copy()
        Ns *= R
    return col.T.reshape(M)


def reg_chirp(c, L, e):
    """c_e = exp(-i pi e^2 / L) from the plan's chirp table."""
    return c[np.asarray(e)]


@pytest.mark.parametrize("kind,n", [(K_DD, 2048), (K_DD, 1024), (K_DD, 512), (K_ND, 1365), (K_DN, 682),
                                    (K_DD, 4096), (K_NN, 2048)])
def test_register_engine_plans_replay_dft(driver, kind, n):
    """Register-engine plans: the power-of-two length (direct when L is a power of two, else the smallest one
    covering the window's convolution), the rotation table and the chirp table; the engine's
    passes replayed on them give the DFT (Bluestein: pre-chirp, forward FFT, kernel product in natural
    order, conjugate, forward FFT, conjugate, post-chirp)."""
    p = plan(driver, kind, n, "register")
    f = p["fwd"]
    L, M = f["L"], f["M"]
    assert f["eng"] == 1 and M == 2 ** f["lgM"] and M >= 512
    assert np.allclose(p["t"], np.exp(-2j * np.pi * np.arange(M // 16) / M), atol=1e-18)
    rng = np.random.default_rng(n + 10 * kind)
    if not f["blue"]:
        assert M == L
        z = rng.standard_normal(L) + 1j * rng.standard_normal(L)
        got = reg_fft(z, p["t"])
        ref = np.fft.fft(z)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        return
    full = f["nin"] == L and f["nout"] == L
    need = 2 * L - 2 if full else max(f["nin"] + f["nout"], p["inv"]["nin"] + p["inv"]["nout"]) - 1
    assert need <= M < 2 * need
    assert len(p["c"]) == L
    assert np.allclose(p["c"], np.exp(-1j * np.pi * ((np.arange(L) ** 2) % (2 * L)) / L), atol=1e-15)
    for tag, bhat in (("fwd", p["b"]), ("inv", p["i"] if len(p["i"]) else p["b"])):
        w = p[tag]
        z = np.zeros(L, complex)
        z[w["in0"]: w["in0"] + w["nin"]] = rng.standard_normal(w["nin"]) + 1j * rng.standard_normal(w["nin"])
        a = np.zeros(M, complex)
        e = np.arange(w["nin"]) + w["in0"]
        a[: w["nin"]] = z[e] * reg_chirp(p["c"], L, e)
        y = np.conj(reg_fft(np.conj(reg_fft(a, p["t"]) * bhat), p["t"]))
        k = np.arange(w["nout"]) + w["out0"]
        got = y[: w["nout"]] * reg_chirp(p["c"], L, k)
        ref = np.fft.fft(z)[k]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (kind, n, tag)


@pytest.mark.parametrize("kind,n,eng,M", [(K_DD, 2048, 1, 4096), (K_ND, 2048, 0, 6144), (K_DN, 2048, 0, 6144),
                                         (K_DD, 1000, 1, 2048), (K_NN, 2048, 1, 2048), (K_NN, 1000, 0, 1000)])
def test_engine_choice(driver, kind, n, eng, M):
    """The planner puts a length on the register engine when it is a power of two >= 512, or needs Bluestein
    and the power-of-two convolution length is no longer than the one the stage engine would pick; otherwise
    the stage engine runs it (ND / DN at 2048: 6144 against 8192)."""
    f = plan(driver, kind, n, "register")["fwd"]
    assert (f["eng"], f["M"]) == (eng, M)


def dd_fold_rows(xa, xb):
    """The DD transform of two rows as the device runs it around its length-(n+1) complex DFT
    (fp_transform.cuh transform_rows, KIND 0): the folded input z(e) = sin(pi e/L)(x_{e-1} + x_{n-e})
    + (x_{e-1} - x_{n-e}) / 2 of both rows as one complex sequence, its DFT Z, and the output pass that
    writes output pair k as out[2k] = s1 (Re Y_0 / 2 + sum_{q=1..k} Re Y_q) and out[2k+1] = -s1 Im Y_{k+1},
    with Y^a_k = (Z_k + conj Z_{L-k}) / 2, Y^b_k = (Z_k - conj Z_{L-k}) / 2i."""
    n = len(xa)
    L = n + 1
    e = np.arange(1, L)
    ta = np.sin(np.pi * np.arange(L) / L)

    def fold(x):
        z = np.zeros(L)
        z[1:] = ta[1:] * (x[e - 1] + x[n - e]) + 0.5 * (x[e - 1] - x[n - e])
        return z

    Z = np.fft.fft(fold(xa) + 1j * fold(xb))
    Zm = Z[(-np.arange(L)) % L]  # Z_{L-k}
    re_a, re_b = 0.5 * (Z.real + Zm.real), 0.5 * (Z.imag + Zm.imag)
    im_a, im_b = 0.5 * (Z.imag - Zm.imag), -0.5 * (Z.real - Zm.real)
    s1 = np.sqrt(2.0 / L)
    K = (n + 1) // 2
    outs = []
    for re, im in ((re_a, im_a), (re_b, im_b)):
        v = re[:K].copy()
        v[0] *= 0.5
        out = np.zeros(n)
        k = np.arange(K)
        out[2 * k] = s1 * np.cumsum(v)
        ko = k[2 * k + 1 < n]
        out[2 * ko + 1] = -s1 * im[ko + 1]
        outs.append(out)
    return outs


@pytest.mark.parametrize("n", [2048, 1000, 97, 8, 5])
def test_dd_fold_output_pairs_replay(n):
    """The DD fold and its output pairs (even outputs from the prefix sum, odd ones from the imaginary
    parts), replayed in numpy around an exact DFT, give the orthonormal DST-I of both rows (the reference's
    PoissonFFT2D_DD, pe/poisson/poisson_fft2d.cpp:19-57), for even and odd row lengths."""
    scipy_fft = pytest.importorskip("scipy.fft")
    rng = np.random.default_rng(n)
    xa, xb = rng.standard_normal(n), rng.standard_normal(n)
    ga, gb = dd_fold_rows(xa, xb)
    for x, got in ((xa, ga), (xb, gb)):
        ref = scipy_fft.dst(x, type=1, norm="ortho")
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), n
