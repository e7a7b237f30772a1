// Host-side planning: FFT stage factorisation, twiddle / chirp / permutation tables, transform
// family tables and rectangle-solver coefficients.
#include "fp_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>

namespace fpb
{

namespace
{
typedef std::complex<long double> cld;
const long double kPi = 3.141592653589793238462643383279502884L;
const double      kRefPi = 3.14159265358979323846;  // the reference's `pi` (base/pch.h:13)

cld root_of_unity(long long num, long long den)  // exp(-2 pi i num / den), exact reduction
{
    num %= den;
    if (num < 0) num += den;
    long double a = -2.0L * kPi * (long double)num / (long double)den;
    return cld(std::cos(a), std::sin(a));
}

// Radix sequence for a 7-smooth length (8s first, then 4, 2, 3, 5, 7); empty if not 7-smooth.
std::vector<int> radices(int m)
{
    std::vector<int> r;
    if (m == 1) return r;
    while (m % 8 == 0) { r.push_back(8); m /= 8; }
    while (m % 4 == 0) { r.push_back(4); m /= 4; }
    while (m % 2 == 0) { r.push_back(2); m /= 2; }
    while (m % 3 == 0) { r.push_back(3); m /= 3; }
    while (m % 5 == 0) { r.push_back(5); m /= 5; }
    while (m % 7 == 0) { r.push_back(7); m /= 7; }
    if (m != 1) r.clear();
    return r;
}

double stage_cost(int R)  // flops per element of one stage (butterfly + twiddle), rough
{
    switch (R)
    {
        case 2: return 5.0;
        case 3: return 9.3;
        case 4: return 8.5;
        case 5: return 13.6;
        case 7: return 19.0;
        default: return 12.3;
    }
}

// Position p of the DIF output holds X[digit_reverse(p)].
std::vector<int> dif_order(const FftDesc& d)
{
    std::vector<int> idx(d.M);
    for (int p = 0; p < d.M; ++p)
    {
        long long k = 0, mult = 1;
        int       pp = p;
        for (int s = 0; s < d.nst; ++s)
        {
            int k1 = pp / d.st[s].S;
            pp -= k1 * d.st[s].S;
            k += (long long)k1 * mult;
            mult *= d.st[s].R;
        }
        idx[p] = (int)k;
    }
    return idx;
}

void host_dft(std::vector<cld>& x)  // natural-order forward DFT, recursive mixed radix (host only)
{
    const int n = (int)x.size();
    if (n <= 1) return;
    int p = 2;
    while (p * p <= n && n % p) ++p;
    if (n % p) p = n;
    const int       m = n / p;
    std::vector<cld> out(n);
    std::vector<std::vector<cld>> sub(p, std::vector<cld>(m));
    for (int r = 0; r < p; ++r)
        for (int k = 0; k < m; ++k) sub[r][k] = x[(size_t)k * p + r];
    for (int r = 0; r < p; ++r) host_dft(sub[r]);
    for (int k = 0; k < n; ++k)
    {
        cld acc = 0;
        for (int r = 0; r < p; ++r) acc += sub[r][k % m] * root_of_unity((long long)r * k, n);
        out[k] = acc;
    }
    x.swap(out);
}

void build_stages(FftDesc& d, const std::vector<int>& rad, std::vector<cld>& tw)
{
    if ((int)rad.size() > kFftMaxStages) throw std::runtime_error("FFT plan: too many stages");
    d.nst = (int)rad.size();
    int B = d.M;
    tw.clear();
    for (int s = 0; s < d.nst; ++s)
    {
        const int R = rad[s], S = B / R;
        d.st[s].R      = R;
        d.st[s].S      = S;
        d.st[s].B      = B;
        d.st[s].tw_off = (int)tw.size();
        for (int b = 0; b < S; ++b) tw.push_back(root_of_unity(b, B));
        B = S;
    }
}
}  // namespace

int kind_of(int bn, int bp)
{
    if (bn == BC_PERIODIC && bp == BC_PERIODIC) return K_PP;
    if (bn == BC_NEUMANN && bp == BC_NEUMANN) return K_NN;
    if (dir_like(bn) && dir_like(bp)) return K_DD;
    if (dir_like(bn) && bp == BC_NEUMANN) return K_DN;
    if (bn == BC_NEUMANN && dir_like(bp)) return K_ND;
    return -1;
}

int fft_length(int kind, int n)
{
    switch (kind)
    {
        case K_DD: return n + 1;
        case K_NN: return n;
        case K_ND:
        case K_DN: return 2 * n + 1;
        default: return n;
    }
}

FftWindow fft_window(int kind, int n, bool inverse)
{
    if (kind == K_ND && inverse) return FftWindow{1, 2 * n, 1, n};  // herm_input 1..2n; outputs X_{j+1}
    if (kind == K_ND || kind == K_DN) return FftWindow{1, n, 1, 2 * n};  // inputs 1..n; X_k, X_{L-k}, k <= n
    const int L = fft_length(kind, n);
    return FftWindow{0, L, 0, L};
}

namespace
{
// Shortest cyclic convolution that is exact for window w of a length-L chirp-z transform.
int window_span(int L, const FftWindow& w)
{
    if (w.in0 == w.out0 && w.nin == L && w.nout == L) return 2 * L - 2;  // the full window: even kernel
    return w.nin + w.nout - 1;
}

// FFT_M of the kernel conj(c_{delta + j}), lags j = -(nin-1) .. nout-1 placed at j mod M, delta =
// out0 - in0; digit-reversed and scaled by 1/M.
std::vector<cld> bluestein_kernel(int L, int M, const FftWindow& w, const FftDesc& d)
{
    std::vector<cld> b(M, cld(0, 0));
    const long long  delta = (long long)w.out0 - w.in0;
    for (long long j = -(long long)(w.nin - 1); j <= (long long)w.nout - 1; ++j)
    {
        long long e = delta + j;  // chirp index; c_e = exp(-i pi e^2 / L) depends on e^2 mod 2L
        long long q = ((e % (2LL * L)) * (e % (2LL * L))) % (2LL * L);
        b[(size_t)(((j % M) + M) % M)] = std::conj(root_of_unity(q, 2LL * L));
    }
    host_dft(b);
    std::vector<int> idx = dif_order(d);
    std::vector<cld> r(M);
    for (int p = 0; p < M; ++p) r[p] = b[idx[p]] / (long double)M;
    return r;
}

void set_window(FftDesc& d, const FftWindow& w)
{
    d.in0  = w.in0;
    d.nin  = w.nin;
    d.out0 = w.out0;
    d.nout = w.nout;
}
}  // namespace

HostFft plan_fft(int L, size_t elem_bytes, size_t smem_limit)
{
    return plan_fft(L, elem_bytes, smem_limit, FftWindow{0, L, 0, L}, FftWindow{0, L, 0, L});
}

namespace
{
// FP_FFT_ENGINE=stage keeps every plan on the stage engine (for comparisons); unset or anything else lets
// the planner pick the register engine where it applies.
bool register_engine_allowed()
{
    const char* e = std::getenv("FP_FFT_ENGINE");
    return !(e && std::string(e) == "stage");
}

// FP_FFT_ENGINE=register: the register engine takes every Bluestein length it can hold, also where its power
// of two is longer than the stage engine's choice
bool register_engine_preferred()
{
    const char* e = std::getenv("FP_FFT_ENGINE");
    return e && std::string(e) == "register";
}

// The stage engine's Bluestein length for a convolution of at least `need` points: the 7-smooth length in
// [need, 1.5 need] with the smallest estimated cost (-1 if none).
int stage_bluestein_length(int need)
{
    int    best      = -1;
    double best_cost = 1e300;
    for (int M = need; M <= need + need / 2; ++M)
    {
        std::vector<int> r = radices(M);
        if (r.empty()) continue;
        double c = 0;
        for (int x : r) c += stage_cost(x);
        c *= M;
        if (c < best_cost)
        {
            best_cost = c;
            best      = M;
        }
    }
    return best;
}

// Natural-order FFT_M of the windowed Bluestein kernel (see bluestein_kernel), scaled by 1/M.
std::vector<cld> bluestein_kernel_natural(int L, int M, const FftWindow& w)
{
    std::vector<cld> b(M, cld(0, 0));
    const long long  delta = (long long)w.out0 - w.in0;
    for (long long j = -(long long)(w.nin - 1); j <= (long long)w.nout - 1; ++j)
    {
        long long e = delta + j;
        long long q = ((e % (2LL * L)) * (e % (2LL * L))) % (2LL * L);
        b[(size_t)(((j % M) + M) % M)] = std::conj(root_of_unity(q, 2LL * L));
    }
    host_dft(b);
    for (auto& x : b) x /= (long double)M;
    return b;
}

// Register-engine plan (fp_fft16.cuh): L a power of two >= kRegMinM (direct), or an L that is not 7-smooth
// (Bluestein) with a power-of-two convolution length. False when neither applies or the buffer and
// tables exceed smem_limit; the stage engine then takes the length.
bool plan_register(int L, size_t elem_bytes, size_t smem_limit, const FftWindow& fw, const FftWindow& iw, HostFft& h)
{
    const bool pow2  = L >= kRegMinM && (L & (L - 1)) == 0;
    const int  max_M = elem_bytes >= 16 ? 8192 : 16384;  // FP64: 512 threads x 128 registers; FP32: 1024 x 64
    int        M     = L;
    if (!pow2)
    {
        if (!radices(L).empty()) return false;  // smooth: the stage engine runs it without Bluestein
        const int need = std::max(window_span(L, fw), window_span(L, iw));
        M              = kRegMinM;
        while (M < need) M *= 2;
        // a power of two longer than the stage engine's own choice (ND / DN windows need 3n - 1: 6144 against
        // 8192 at n = 2048) costs more than the register engine saves
        const int stage_M = stage_bluestein_length(need);
        if (stage_M > 0 && M > stage_M && !register_engine_preferred()) return false;
    }
    if (M > max_M) return false;
    const size_t elems = (size_t)reg_buf_elems(M) + M / 16 + (pow2 ? 0 : reg_chirp_entries(L));
    if (elems * elem_bytes > smem_limit) return false;
    h.d      = FftDesc{};
    h.d.L    = L;
    h.d.M    = M;
    h.d.blue = pow2 ? 0 : 1;
    h.d.eng  = 1;
    h.d.pad  = kRegPad;
    int lg   = 0;
    while ((1 << lg) < M) ++lg;
    h.d.lgM = lg;
    h.d.nst = 0;
    h.tw.resize(M / 16);
    for (int m = 0; m < M / 16; ++m) h.tw[m] = root_of_unity(m, M);
    h.d_inv = h.d;
    if (pow2)
    {
        set_window(h.d, FftWindow{0, L, 0, L});
        set_window(h.d_inv, FftWindow{0, L, 0, L});
        return true;
    }
    set_window(h.d, fw);
    set_window(h.d_inv, iw);
    h.chirp.resize(L);  // c_e = exp(-i pi e^2 / L)
    for (int e = 0; e < L; ++e) h.chirp[e] = root_of_unity(((long long)e * e) % (2LL * L), 2LL * L);
    h.bhat = bluestein_kernel_natural(L, M, fw);
    if (fw.in0 != iw.in0 || fw.nin != iw.nin || fw.out0 != iw.out0 || fw.nout != iw.nout)
        h.bhat_inv = bluestein_kernel_natural(L, M, iw);
    return true;
}
}  // namespace

HostFft plan_fft(int L, size_t elem_bytes, size_t smem_limit, FftWindow fw, FftWindow iw, bool allow_register,
                 bool allow_global)
{
    HostFft h;
    if (allow_register && register_engine_allowed() && plan_register(L, elem_bytes, smem_limit, fw, iw, h)) return h;
    h.d.L   = L;
    h.d.eng = 0;
    h.d.pad = 3;
    std::vector<int> rad = radices(L);
    if (!rad.empty() || L == 1)
    {
        h.d.M    = L;
        h.d.blue = 0;
        set_window(h.d, FftWindow{0, L, 0, L});
        build_stages(h.d, rad, h.tw);
        std::vector<int> idx = dif_order(h.d);
        h.perm.assign(L, 0);
        for (int p = 0; p < L; ++p) h.perm[idx[p]] = p;
        h.d_inv = h.d;
    }
    else
    {
        for (const FftWindow& w : {fw, iw})
            if (w.in0 < 0 || w.nin < 1 || w.in0 + w.nin > L || w.out0 < 0 || w.nout < 1 || w.out0 + w.nout > L)
                throw std::runtime_error("FFT plan: window outside the transform");
        // Smallest-cost 7-smooth M covering both windows' convolutions.
        const int need = std::max(window_span(L, fw), window_span(L, iw));
        const int best = stage_bluestein_length(need);
        if (best < 0) throw std::runtime_error("FFT plan: no Bluestein length");
        h.d.M    = best;
        h.d.blue = 1;
        build_stages(h.d, radices(best), h.tw);
        h.d_inv = h.d;
        set_window(h.d, fw);
        set_window(h.d_inv, iw);
        h.chirp.resize(L);
        for (int n = 0; n < L; ++n) h.chirp[n] = root_of_unity(((long long)n * n) % (2LL * L), 2LL * L);
        h.bhat = bluestein_kernel(L, best, fw, h.d);
        if (fw.in0 != iw.in0 || fw.nin != iw.nin || fw.out0 != iw.out0 || fw.nout != iw.nout)
            h.bhat_inv = bluestein_kernel(L, best, iw, h.d);
    }
    if ((size_t)fft_buf_elems(h.d.M) * elem_bytes > smem_limit && allow_global)
    {
        h.d.eng     = 2;
        h.d_inv.eng = 2;
    }
    else if ((size_t)fft_buf_elems(h.d.M) * elem_bytes > smem_limit)
        throw std::runtime_error("transform length " + std::to_string(L) + " needs " +
                                 std::to_string((size_t)fft_buf_elems(h.d.M) * elem_bytes) +
                                 " bytes of shared memory, more than this build supports");
    return h;
}

KindTables kind_tables(int kind, int n)
{
    KindTables t;
    const double pi = kRefPi;
    switch (kind)
    {
        case K_DD:  // poisson_fft2d.cpp:22; folding weights of the length-(n+1) DST-I
            t.s1 = std::sqrt(2.0 / (1. + n));
            t.a.resize(n + 1);
            for (int j = 0; j <= n; ++j) t.a[j] = (double)std::sin(kPi * (long double)j / (long double)(n + 1));
            break;
        case K_NN:                                             // poisson_fft2d.cpp:81-90
            t.s1 = std::sqrt(2.0 / n);
            t.s2 = std::sqrt(1.0 / n);
            t.a.resize(n);
            t.b.resize(n);
            for (int j = 0; j < n; j++)
            {
                t.a[j] = std::cos(pi * (j + 1.) / n / 2);
                t.b[j] = std::sin(pi * (j + 1.) / n / 2);
            }
            t.c.resize(n);  // Makhoul post-twiddle exp(-i pi m / 2n)
            for (int m = 0; m < n; ++m) t.c[m] = root_of_unity(m, 4LL * n);
            break;
        case K_ND:  // poisson_fft2d.cpp:157-165
            t.s1 = std::sqrt(4. / (2. * n + 1.));
            t.a.resize(n);
            t.b.resize(n);
            for (int j = 0; j < n; j++)
            {
                t.a[j] = std::cos(2. * n * pi * (j + 1.) / (2. * n + 1.));
                t.b[j] = std::sin(2. * n * pi * (j + 1.) / (2. * n + 1.));
            }
            break;
        case K_DN: t.s1 = std::sqrt(4. / (2. * n + 1.)); break;  // poisson_fft2d.cpp:227
        case K_PP:                                                 // poisson_fft2d.cpp:390-397
            t.s1 = std::sqrt(2.0 / n);
            t.a.resize(n);
            t.b.resize(n);
            for (int j = 0; j < n; j++)
            {
                t.a[j] = std::cos(pi * (2.0 * j + 1.0) / 4.0);
                t.b[j] = std::sin(pi * (2.0 * j + 1.0) / 4.0);
            }
            break;
        default: throw std::runtime_error("unknown transform family");
    }
    return t;
}

std::vector<double> cal_lambda(int n, int bn, int bp)
{
    const double        pi = kRefPi;
    std::vector<double> lam(n);
    for (int i = 1; i <= n; i++)
    {
        double v;
        if (bn == BC_PERIODIC && bp == BC_PERIODIC) v = -2.0 * std::cos(2.0 * pi / n * std::floor(i / 2.0));
        else if (bn == BC_NEUMANN && bp == BC_NEUMANN) v = -2.0 * std::cos(pi / n * i);
        else if (dir_like(bn) && dir_like(bp)) v = +2.0 * std::cos(pi / (n + 1) * i);
        else if ((dir_like(bn) && bp == BC_NEUMANN) || (bn == BC_NEUMANN && dir_like(bp)))
            v = -2.0 * std::cos(2.0 * pi * i / (2 * n + 1));
        else throw std::runtime_error("unsupported boundary pair");
        lam[i - 1] = v;
    }
    return lam;
}

std::vector<double> x_diag(int ny, double hx, double hy, int bn, int bp)
{
    std::vector<double> lam = cal_lambda(ny, bn, bp);
    std::vector<double> d(ny);
    for (int j = 0; j < ny; j++) d[j] = -2.0 + hx * hx / hy / hy * (lam[j] - 2.0);
    return d;
}

}  // namespace fpb
