// Oracle-only real-to-complex DFT behind the fftw3.h stand-in (see fftw3.h for the semantics).
//
// TEST INFRASTRUCTURE: linked only into oracle/_ref (the reference's own sources built for CPU
// parity and the CPU baseline). Algorithm, restated from the textbook DFT:
//   * complex DFT of length m by iterative Stockham auto-sort stages, one stage per prime-power
//     factor (radices 4, 2, 3, 5, 7 and any other small prime by direct summation);
//   * when m has a prime factor above 61, Bluestein's chirp-z transform on a power-of-two
//     convolution length, with the chirp exp(-i*pi*n^2/m) evaluated from (n^2 mod 2m) so it keeps
//     full double accuracy for every n;
//   * real input of even length n is packed as n/2 complex points and unpacked with the
//     standard split formula; odd n goes through the complex transform directly.
// fftw_execute_dft_r2c is reentrant (the reference calls it from OpenMP threads on one plan):
// all scratch lives in thread_local buffers.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace
{
typedef std::complex<double> cd;
const long double kPi = 3.141592653589793238462643383279502884L;

cd unit_root(long long num, long long den)  // exp(-2*pi*i*num/den), reduced exactly
{
    num %= den;
    if (num < 0) num += den;
    long double a = -2.0L * kPi * (long double)num / (long double)den;
    return cd((double)std::cos(a), (double)std::sin(a));
}

struct Stage
{
    int             radix;
    int             ns;  // product of the radices of earlier stages
    std::vector<cd> tw;  // tw[jj*radix + r] = exp(-2 pi i r jj / (ns*radix))
    std::vector<cd> w;   // w[k] = exp(-2 pi i k / radix)
};

struct ComplexPlan
{
    int                m = 0;
    std::vector<Stage> stages;
    // Bluestein
    bool               blue = false;
    int                M    = 0;
    std::vector<cd>    chirp;  // exp(-i pi n^2 / m), n < m
    std::vector<cd>    bhat;   // FFT_M of the conjugate chirp kernel, divided by M
    ComplexPlan*       inner = nullptr;

    ~ComplexPlan() { delete inner; }
};

std::vector<int> factor(int m)
{
    std::vector<int> f;
    while (m % 4 == 0) { f.push_back(4); m /= 4; }
    while (m % 2 == 0) { f.push_back(2); m /= 2; }
    for (int p = 3; (long long)p * p <= m; p += 2)
        while (m % p == 0) { f.push_back(p); m /= p; }
    if (m > 1) f.push_back(m);
    return f;
}

void build_stages(ComplexPlan* pl, const std::vector<int>& radices)
{
    int ns = 1;
    for (int r : radices)
    {
        Stage s;
        s.radix = r;
        s.ns    = ns;
        s.tw.resize((size_t)ns * r);
        for (int jj = 0; jj < ns; ++jj)
            for (int q = 0; q < r; ++q) s.tw[(size_t)jj * r + q] = unit_root((long long)q * jj, (long long)ns * r);
        s.w.resize(r);
        for (int k = 0; k < r; ++k) s.w[k] = unit_root(k, r);
        pl->stages.push_back(std::move(s));
        ns *= r;
    }
}

ComplexPlan* make_complex_plan(int m);

void run_complex(const ComplexPlan* pl, cd* data, std::vector<cd>& work);

ComplexPlan* make_complex_plan(int m)
{
    ComplexPlan* pl = new ComplexPlan();
    pl->m           = m;
    std::vector<int> f = factor(m);
    int              maxp = 1;
    for (int p : f) maxp = p > maxp ? p : maxp;
    if (maxp <= 61)
    {
        build_stages(pl, f);
        return pl;
    }
    pl->blue = true;
    int M    = 1;
    while (M < 2 * m - 1) M <<= 1;
    pl->M = M;
    pl->chirp.resize(m);
    for (int n = 0; n < m; ++n)
    {
        long long nn = ((long long)n * n) % (2LL * m);
        pl->chirp[n] = unit_root(nn, 2LL * m);  // exp(-2 pi i nn/(2m)) = exp(-i pi n^2/m)
    }
    pl->inner = make_complex_plan(M);
    std::vector<cd> b(M, cd(0, 0));
    for (int n = 0; n < m; ++n) b[n] = std::conj(pl->chirp[n]);
    for (int n = 1; n < m; ++n) b[M - n] = std::conj(pl->chirp[n]);
    std::vector<cd> work;
    run_complex(pl->inner, b.data(), work);
    pl->bhat.resize(M);
    for (int k = 0; k < M; ++k) pl->bhat[k] = b[k] / (double)M;
    return pl;
}

inline void small_dft(cd* v, int r, const cd* w)
{
    if (r == 2)
    {
        cd a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
        return;
    }
    if (r == 4)
    {
        cd a = v[0], b = v[1], c = v[2], d = v[3];
        cd s0 = a + c, s1 = a - c, s2 = b + d, s3 = b - d;
        cd s3j(s3.imag(), -s3.real());  // -i * s3
        v[0] = s0 + s2;
        v[1] = s1 + s3j;
        v[2] = s0 - s2;
        v[3] = s1 - s3j;
        return;
    }
    cd out[64];
    for (int k = 0; k < r; ++k)
    {
        cd acc = 0;
        for (int q = 0; q < r; ++q) acc += v[q] * w[(size_t)((long long)q * k % r)];
        out[k] = acc;
    }
    for (int k = 0; k < r; ++k) v[k] = out[k];
}

void run_complex(const ComplexPlan* pl, cd* data, std::vector<cd>& work)
{
    const int m = pl->m;
    if (!pl->blue)
    {
        if ((int)work.size() < m) work.resize(m);
        cd* src = data;
        cd* dst = work.data();
        for (const Stage& s : pl->stages)
        {
            const int R  = s.radix;
            const int nr = m / R;
            const int Ns = s.ns;
            cd        v[64];
            for (int j = 0; j < nr; ++j)
            {
                const int jj = j % Ns;
                const cd* tw = &s.tw[(size_t)jj * R];
                for (int q = 0; q < R; ++q) v[q] = src[j + q * nr] * tw[q];
                small_dft(v, R, s.w.data());
                const int idx = (j / Ns) * Ns * R + jj;
                for (int q = 0; q < R; ++q) dst[idx + q * Ns] = v[q];
            }
            cd* t = src;
            src   = dst;
            dst   = t;
        }
        if (src != data)
            for (int k = 0; k < m; ++k) data[k] = src[k];
        return;
    }
    // Bluestein: X_k = conj(c_k)... with c_n = exp(-i pi n^2/m):
    //   X_k = c_k * sum_n (x_n c_n) * conj(c_{k-n})
    const int                    M = pl->M;
    thread_local std::vector<cd> a;
    thread_local std::vector<cd> w2;
    a.assign(M, cd(0, 0));
    for (int n = 0; n < m; ++n) a[n] = data[n] * pl->chirp[n];
    run_complex(pl->inner, a.data(), w2);
    for (int k = 0; k < M; ++k) a[k] = std::conj(a[k] * pl->bhat[k]);
    run_complex(pl->inner, a.data(), w2);  // conj(FFT(conj(.))) = M * IFFT(.)
    for (int k = 0; k < m; ++k) data[k] = std::conj(a[k]) * pl->chirp[k];
}

}  // namespace

struct fp_oracle_r2c_plan
{
    int              n    = 0;
    bool             even = false;
    ComplexPlan*     cp   = nullptr;
    std::vector<cd>  post;  // exp(-2 pi i k / n), k = 0..n/2 (even n only)
    ~fp_oracle_r2c_plan() { delete cp; }
};

extern "C" fftw_plan fftw_plan_dft_r2c_1d(int n, double*, fftw_complex*, unsigned)
{
    fftw_plan p = new fp_oracle_r2c_plan();
    p->n        = n;
    p->even     = (n % 2 == 0) && n >= 2;
    if (p->even)
    {
        p->cp = make_complex_plan(n / 2);
        p->post.resize(n / 2 + 1);
        for (int k = 0; k <= n / 2; ++k) p->post[k] = unit_root(k, n);
    }
    else
    {
        p->cp = make_complex_plan(n);
    }
    return p;
}

extern "C" void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out)
{
    thread_local std::vector<cd> z;
    thread_local std::vector<cd> work;
    const int                    n = p->n;
    if (p->even)
    {
        const int m = n / 2;
        if ((int)z.size() < m) z.resize(m);
        for (int k = 0; k < m; ++k) z[k] = cd(in[2 * k], in[2 * k + 1]);
        run_complex(p->cp, z.data(), work);
        for (int k = 0; k <= m; ++k)
        {
            cd zk  = z[k % m];
            cd zmk = std::conj(z[(m - k) % m]);
            cd e   = 0.5 * (zk + zmk);
            cd o   = cd(0, -0.5) * (zk - zmk);
            cd X   = e + p->post[k] * o;
            out[k][0] = X.real();
            out[k][1] = X.imag();
        }
    }
    else
    {
        if ((int)z.size() < n) z.resize(n);
        for (int k = 0; k < n; ++k) z[k] = cd(in[k], 0.0);
        run_complex(p->cp, z.data(), work);
        for (int k = 0; k <= n / 2; ++k)
        {
            out[k][0] = z[k].real();
            out[k][1] = z[k].imag();
        }
    }
}

extern "C" void fftw_destroy_plan(fftw_plan p) { delete p; }
