// Device-resident transform and rectangle (PoissonSolver2D) plans.
#include "fp_chase.cuh"
#include "fp_internal.h"

#include <algorithm>
#include <mutex>

namespace fpb
{

size_t max_dynamic_smem()
{
    static size_t v = [] {
        int dev = 0, optin = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return (size_t)48 * 1024;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            return (size_t)48 * 1024;
        return (size_t)optin - 1024;  // room for the kernel's static shared arrays
    }();
    return v;
}

namespace
{
template <typename T> std::vector<T> convert(const std::vector<double>& v)
{
    return std::vector<T>(v.begin(), v.end());
}
template <typename T2> std::vector<T2> convert_c(const std::vector<std::complex<long double>>& v)
{
    std::vector<T2> r(v.size());
    for (size_t i = 0; i < v.size(); ++i)
    {
        r[i].x = (decltype(r[i].x))v[i].real();
        r[i].y = (decltype(r[i].y))v[i].imag();
    }
    return r;
}

template <typename T, int K, int I> void launch_k(const TransformArgs<T>& a, long long rows, int threads, size_t smem,
                                                  cudaStream_t s)
{
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(k_transform<T, K, I>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)max_dynamic_smem());
    });
    const long long grid = FamilyTraits<K, I>::kPairRows ? (rows + 1) / 2 : rows;
    if (grid <= 0) return;
    k_transform<T, K, I><<<(unsigned)grid, threads, smem, s>>>(a);
    FPB_CHECK_LAUNCH();
}
}  // namespace

template <typename T> DevTransform<T>::DevTransform(int kind_, int n_) : kind(kind_), n(n_)
{
    if (n < 2) throw Error(1, "row length must be at least 2");
    if (kind == K_PP && (n % 2)) throw Error(1, "periodic transform needs an even length");
    const int L = r2c_length(kind, n);
    HostFft   h;
    try
    {
        h = plan_fft(L, sizeof(T2), max_dynamic_smem());
    }
    catch (const std::runtime_error& e)
    {
        throw Error(3, e.what());
    }
    fd = h.d;
    tw = upload(convert_c<T2>(h.tw));
    if (fd.blue)
    {
        chirp = upload(convert_c<T2>(h.chirp));
        bhat  = upload(convert_c<T2>(h.bhat));
    }
    else
    {
        perm = upload(h.perm);
    }
    KindTables kt = kind_tables(kind, n);
    if (!kt.a.empty())
    {
        ta = upload(convert<T>(kt.a));
        tb = upload(convert<T>(kt.b));
    }
    s1      = (T)kt.s1;
    s2      = (T)kt.s2;
    threads = std::min(512, std::max(64, ((fd.M / 8 + 31) / 32) * 32));
    smem    = (size_t)fd.M * sizeof(T2);
}

template <typename T> void DevTransform<T>::run(const T* in, T* out, long long rows, bool inverse, cudaStream_t s) const
{
    TransformArgs<T> a;
    a.in    = in;
    a.out   = out;
    a.rows  = rows;
    a.n     = n;
    a.fd    = fd;
    a.ft    = FftTables<T2>{tw.as<T2>(), chirp.as<T2>(), bhat.as<T2>(), perm.as<int>()};
    a.ta    = ta.as<T>();
    a.tb    = tb.as<T>();
    a.s1    = s1;
    a.s2    = s2;
    const int inv = inverse ? 1 : 0;
#define FPB_CASE(K)                                                                                        \
    case K:                                                                                                \
        if (inv) launch_k<T, K, 1>(a, rows, threads, smem, s);                                              \
        else launch_k<T, K, 0>(a, rows, threads, smem, s);                                                  \
        break;
    switch (kind)
    {
        FPB_CASE(0)
        FPB_CASE(1)
        FPB_CASE(2)
        FPB_CASE(3)
        FPB_CASE(4)
        default: throw Error(1, "unknown transform family");
    }
#undef FPB_CASE
}

namespace
{
// Thomas coefficients per (row i, wavenumber j), computed with the reference's divisions
// (chasing_method_base.cpp:34-46 / :126-131): see fp_chase.cuh for the table's meaning.
void chase_table(int nx, int ny, const std::vector<double>& d, bool start_neu, bool end_neu, std::vector<double>& c)
{
    c.assign((size_t)nx * ny, 0.0);
    for (int j = 0; j < ny; ++j)
    {
        const double dj = d[j];
        double       cp = start_neu ? 1.0 / (dj + 1.0) : 1.0 / dj;
        c[j]            = cp;
        for (int i = 1; i < nx - 1; ++i)
        {
            cp                    = 1.0 / (dj - cp);
            c[(size_t)i * ny + j] = cp;
        }
        if (nx >= 2) c[(size_t)(nx - 1) * ny + j] = end_neu ? 1.0 / (dj + 1.0 - cp) : 1.0 / (dj - cp);
    }
}
// Sherman-Morrison special solutions z1 = T^-1 e_0, z2 = T^-1 e_{n-1} of the Dirichlet system
// (chasing_method_base.cpp:200-231).
void periodic_tables(int nx, int ny, const std::vector<double>& d, std::vector<double>& z1, std::vector<double>& z2)
{
    z1.assign((size_t)nx * ny, 0.0);
    z2.assign((size_t)nx * ny, 0.0);
    std::vector<double> c(nx), y(nx), u(nx);
    for (int j = 0; j < ny; ++j)
    {
        const double dj = d[j];
        for (int which = 0; which < 2; ++which)
        {
            for (int i = 0; i < nx; ++i) u[i] = (which == 0) ? (i == 0 ? 1.0 : 0.0) : (i == nx - 1 ? 1.0 : 0.0);
            c[0] = 1.0 / dj;
            for (int i = 1; i < nx - 1; i++) c[i] = 1.0 / (dj - c[i - 1]);
            y[0] = u[0] / dj;
            for (int i = 1; i < nx - 1; i++) y[i] = (u[i] - y[i - 1]) / (dj - c[i - 1]);
            y[nx - 1]                     = (u[nx - 1] - y[nx - 2]) / (dj - c[nx - 2]);
            std::vector<double>& z        = which == 0 ? z1 : z2;
            double               x        = y[nx - 1];
            z[(size_t)(nx - 1) * ny + j] = x;
            for (int i = nx - 2; i >= 0; i--)
            {
                x                     = y[i] - c[i] * x;
                z[(size_t)i * ny + j] = x;
            }
        }
    }
}
}  // namespace

template <typename T> DevRect<T>::DevRect(int nx_, int ny_, double hx_, double hy_, const int* bc_)
    : nx(nx_), ny(ny_), hx(hx_), hy(hy_)
{
    for (int f = 0; f < 4; ++f) bc[f] = bc_[f];
    if (nx < 2 || ny < 2) throw Error(1, "each subdomain needs at least 2 cells per direction");
    if (!(hx > 0) || !(hy > 0)) throw Error(1, "grid spacings must be positive");
    const int kind = kind_of(bc[YNEG], bc[YPOS]);
    if (kind < 0) throw Error(1, "unsupported y boundary pair");
    const bool xp = bc[XNEG] == BC_PERIODIC && bc[XPOS] == BC_PERIODIC;
    if (!xp && (bc[XNEG] == BC_PERIODIC || bc[XPOS] == BC_PERIODIC || bc[XNEG] == BC_NULL || bc[XPOS] == BC_NULL))
        throw Error(1, "unsupported x boundary pair");
    tr.reset(new DevTransform<T>(kind, ny));
    periodic_x = xp;
    singular   = !(dir_like(bc[0]) || dir_like(bc[1]) || dir_like(bc[2]) || dir_like(bc[3]));
    std::vector<double> d = x_diag(ny, hx, hy, bc[YNEG], bc[YPOS]);
    std::vector<double> c;
    chase_table(nx, ny, d, !xp && bc[XNEG] == BC_NEUMANN, !xp && bc[XPOS] == BC_NEUMANN, c);
    ctab = upload(convert<T>(c));
    if (periodic_x)
    {
        std::vector<double> a, b;
        periodic_tables(nx, ny, d, a, b);
        z1 = upload(convert<T>(a));
        z2 = upload(convert<T>(b));
    }
}

template <typename T> void DevRect<T>::solve(T* f, long long batch, cudaStream_t s) const
{
    if (batch <= 0) return;
    tr->run(f, f, batch * nx, false, s);
    const long long nthreads = batch * ny;
    const int       block    = 128;
    k_chase<T><<<(unsigned)((nthreads + block - 1) / block), block, 0, s>>>(f, nx, ny, batch, ctab.as<T>(),
                                                                           z1.as<T>(), z2.as<T>(),
                                                                           periodic_x ? 1 : 0, singular ? 1 : 0);
    FPB_CHECK_LAUNCH();
    tr->run(f, f, batch * nx, true, s);
}

template struct DevTransform<double>;
template struct DevTransform<float>;
template struct DevRect<double>;
template struct DevRect<float>;

}  // namespace fpb
