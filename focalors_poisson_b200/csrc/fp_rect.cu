// Device-resident transform and rectangle (PoissonSolver2D) plans.
#include "fp_chase.cuh"
#include "fp_internal.h"

#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <type_traits>

namespace fpb
{

// Largest dynamic shared memory a CTA may opt into on the current device, less room for static arrays.
// Cached per device: a process may drive several GPUs.
size_t max_dynamic_smem()
{
    static std::mutex mu;
    static size_t     cache[kMaxDevices] = {};
    int               dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return (size_t)48 * 1024;
    std::lock_guard<std::mutex> lk(mu);
    if (!cache[dev])
    {
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            return (size_t)48 * 1024;
        cache[dev] = (size_t)optin - 1024;  // room for the kernel's static shared arrays
    }
    return cache[dev];
}

// CTAs of `threads` threads and `smem` dynamic shared memory that fit on the current device at once
// (SMs x resident CTAs per SM), cached per (device, kernel, shape).
long long resident_ctas(const void* func, int threads, size_t smem)
{
    static std::mutex                                                     mu;
    static std::map<std::tuple<int, const void*, int, size_t>, long long> cache;
    int                                                                   dev = 0;
    FPB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto                        key = std::make_tuple(dev, func, threads, smem);
    auto                        it  = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0, sms = 0;
    FPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem));
    FPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long v = (long long)std::max(1, per_sm) * std::max(1, sms);
    cache[key]        = v;
    return v;
}

// Function attributes are per device: the opt-in to max_dynamic_smem() is made once per (device, kernel).
void allow_max_dynamic_smem(const void* func)
{
    static std::mutex                             mu;
    static std::set<std::pair<int, const void*>> done;
    int                                           dev = 0;
    FPB_CUDA(cudaGetDevice(&dev));
    const size_t smem = max_dynamic_smem();
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({dev, func})) return;
    FPB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done.insert({dev, func});
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

// One run of rows through k_b_xform with the plan's arguments by value (PV): one CTA per item on the stage
// engine; on the register engine as many CTAs as fit on the GPU at once, each looping over items (its
// tables are loaded once per CTA); a register-engine plan of length kXformStaticM runs k_xform_rc.
template <typename T, int K, int I, typename TIO, int ENG>
void launch_k(const DstSeg& one, const XformArgs<T>& ha, long long rows, int threads, size_t smem, cudaStream_t s,
              long long gctas = 0)
{
    const long long items = FamilyTraits<K, I>::kPairRows ? (rows + 1) / 2 : rows;
    if (items <= 0) return;
    if constexpr (ENG == 1)
    {
        if (ha.fd.M == kXformStaticM)
        {
            const void* fn = (const void*)k_xform_rc<T, K, I, TIO, TIO, false, kXformStaticM>;
            allow_max_dynamic_smem(fn);
            const long long grid = std::min<long long>(items, resident_ctas(fn, threads, smem));
            k_xform_rc<T, K, I, TIO, TIO, false, kXformStaticM>
                <<<(unsigned)grid, threads, smem, s>>>(nullptr, nullptr, 1, items, one, ha);
            FPB_CHECK_LAUNCH();
            return;
        }
    }
    const void* fn = (const void*)k_b_xform<T, K, I, TIO, TIO, false, ENG, true>;
    allow_max_dynamic_smem(fn);
    const long long grid = ENG == 1   ? std::min<long long>(items, resident_ctas(fn, threads, smem))
                           : ENG == 2 ? std::min<long long>(items, gctas)  // the CTAs the global buffers hold
                                      : items;
    k_b_xform<T, K, I, TIO, TIO, false, ENG, true>
        <<<(unsigned)grid, threads, smem, s>>>(nullptr, nullptr, 1, items, nullptr, one, ha);
    FPB_CHECK_LAUNCH();
}
}  // namespace

template <typename T>
DevTransform<T>::DevTransform(int kind_, int n_, bool allow_register, bool allow_global) : kind(kind_), n(n_)
{
    if (n < 2) throw Error(1, "row length must be at least 2");
    if (kind == K_PP && (n % 2)) throw Error(1, "periodic transform needs an even length");
    const int L = fft_length(kind, n);
    HostFft   h;
    try
    {
        h = plan_fft(L, sizeof(T2), max_dynamic_smem(), fft_window(kind, n, false), fft_window(kind, n, true),
                     allow_register, allow_global);
    }
    catch (const std::runtime_error& e)
    {
        throw Error(3, e.what());
    }
    fd     = h.d;
    fd_inv = h.d_inv;
    tw     = upload(convert_c<T2>(h.tw));
    if (fd.blue)
    {
        chirp = upload(convert_c<T2>(h.chirp));
        bhat  = upload(convert_c<T2>(h.bhat));
        if (!h.bhat_inv.empty()) bhat_inv = upload(convert_c<T2>(h.bhat_inv));
    }
    else
    {
        perm = upload(h.perm);
    }
    std::vector<int4> st(fd.nst);
    for (int s = 0; s < fd.nst; ++s) st[s] = make_int4(fd.st[s].R, fd.st[s].S, fd.st[s].B, fd.st[s].tw_off);
    stages        = upload(st);
    KindTables kt = kind_tables(kind, n);
    if (!kt.a.empty())
    {
        ta = upload(convert<T>(kt.a));
        tb = upload(convert<T>(kt.b));
    }
    if (!kt.c.empty()) tc = upload(convert_c<T2>(kt.c));
    s1      = (T)kt.s1;
    s2      = (T)kt.s2;
    const int K_scan = (n + 1) / 2;  // DD prefix-sum arrays: 2K values, in the buffer's tail when it fits
    int       E, tail;                // shared-memory elements; free slots past element L-1 of the buffer
    if (fd.eng == 1)
    {
        threads = fd.M / 16;
        E       = reg_smem_elems(fd);
        tail    = reg_buf_elems(fd.M) - reg_slot(fd.L);
    }
    else
    {
        threads = std::min(512, std::max(64, ((fd.M / 16 + 31) / 32) * 32));
        E       = fft_buf_elems(fd.M);
        tail    = E - fft_slot(fd.L);
    }
    smem = (size_t)E * sizeof(T2) + ((kind == K_DD && tail < K_scan) ? (size_t)2 * K_scan * sizeof(T) : 0);
    if (fd.eng == 2)
    {
        // per CTA: the buffer, then the DD scan arrays (2K values of T in K + 1 complex slots); two CTAs per SM
        int dev = 0, sms = 148;
        FPB_CUDA(cudaGetDevice(&dev));
        FPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        gstride = ((long long)E + K_scan + 1 + 7) & ~7LL;
        gctas   = 2 * sms;
        gscratch.alloc((size_t)gctas * gstride * sizeof(T2));
        smem = 0;
    }
    hargs[0] = args(false);
    hargs[1] = args(true);
    if (smem > max_dynamic_smem()) throw Error(3, "transform of length " + std::to_string(n) + " needs more shared memory than a CTA has");
}

template <typename T> XformArgs<T> DevTransform<T>::args(bool inverse) const
{
    XformArgs<T> a{};
    const bool   inv_tab = inverse && bhat_inv.bytes() > 0;
    a.n  = n;
    a.fd = inverse ? fd_inv : fd;
    a.ft = FftTables<T2>{tw.as<T2>(), chirp.as<T2>(), (inv_tab ? bhat_inv : bhat).template as<T2>(), perm.as<int>(),
                         stages.as<int4>()};
    a.tc = tc.as<T2>();
    a.ta = ta.as<T>();
    a.tb = tb.as<T>();
    a.s1      = s1;
    a.s2      = s2;
    a.gbuf    = gscratch.as<T2>();
    a.gstride = gstride;
    return a;
}

template <typename T>
template <typename TIO>
void DevTransform<T>::run_io(const TIO* in, TIO* out, long long rows, bool inverse, cudaStream_t s) const
{
    if (rows > (long long)INT_MAX) throw Error(3, "more than 2^31 rows in one transform call");
    const DstSeg        a{in, out, (int)rows, 0};
    const int           inv = inverse ? 1 : 0;
    const XformArgs<T>& d   = hargs[inv];
#define FPB_CASE(K)                                                                                        \
    case K:                                                                                                \
        if (fd.eng == 1)                                                                                   \
        {                                                                                                  \
            if (inv) launch_k<T, K, 1, TIO, 1>(a, d, rows, threads, smem, s);                                  \
            else launch_k<T, K, 0, TIO, 1>(a, d, rows, threads, smem, s);                                      \
        }                                                                                                  \
        else if (fd.eng == 2)                                                                              \
        {                                                                                                  \
            if (inv) launch_k<T, K, 1, TIO, 2>(a, d, rows, threads, smem, s, gctas);                           \
            else launch_k<T, K, 0, TIO, 2>(a, d, rows, threads, smem, s, gctas);                               \
        }                                                                                                  \
        else if (inv) launch_k<T, K, 1, TIO, 0>(a, d, rows, threads, smem, s);                                 \
        else launch_k<T, K, 0, TIO, 0>(a, d, rows, threads, smem, s);                                          \
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
// Partition-chase tables for the interior rows (kChunk-1 of them) of a chunk: [type][r][j] Thomas
// factors c, spikes g = T^-1 e_first and h = T^-1 e_last, and [type][4][j] end values
// (g_first, g_last, h_first, h_last). Type 0 is the first chunk (x- Neumann change on its first row).
void partition_tables(int ny, const std::vector<double>& d, bool start_neu, std::vector<double>& c,
                      std::vector<double>& g, std::vector<double>& h, std::vector<double>& ends)
{
    const int Li = kChunk - 1;
    c.assign((size_t)2 * Li * ny, 0.0);
    g.assign((size_t)2 * Li * ny, 0.0);
    h.assign((size_t)2 * Li * ny, 0.0);
    ends.assign((size_t)2 * 4 * ny, 0.0);
    std::vector<double> cc(Li), y(Li), x(Li);
    for (int typ = 0; typ < 2; ++typ)
        for (int j = 0; j < ny; ++j)
        {
            const double dj = d[j];
            cc[0]           = (typ == 0 && start_neu) ? 1.0 / (dj + 1.0) : 1.0 / dj;
            for (int r = 1; r < Li; ++r) cc[r] = 1.0 / (dj - cc[r - 1]);
            for (int r = 0; r < Li; ++r) c[((size_t)typ * Li + r) * ny + j] = cc[r];
            for (int which = 0; which < 2; ++which)
            {
                double prev = 0;
                for (int r = 0; r < Li; ++r)
                {
                    const double rhs = (which == 0) ? (r == 0 ? 1.0 : 0.0) : (r == Li - 1 ? 1.0 : 0.0);
                    prev             = (rhs - prev) * cc[r];
                    y[r]             = prev;
                }
                x[Li - 1] = y[Li - 1];
                for (int r = Li - 2; r >= 0; --r) x[r] = y[r] - cc[r] * x[r + 1];
                std::vector<double>& dst = which == 0 ? g : h;
                for (int r = 0; r < Li; ++r) dst[((size_t)typ * Li + r) * ny + j] = x[r];
                ends[((size_t)typ * 4 + 2 * which + 0) * ny + j] = x[0];
                ends[((size_t)typ * 4 + 2 * which + 1) * ny + j] = x[Li - 1];
            }
        }
}
}  // namespace

// Thomas factors of the separator system of the partition chase (fp_chase.cuh), which depend on the
// wavenumber only: for rows p < pmax taken as not last, cp[p] = up / den_p and iden[p] = 1 / den_p with
// den_p = diag_p - lower_p cp[p-1]; the last row of a given P is formed in the kernel from cp[P-2].
void separator_factors(int ny, int pmax, const std::vector<double>& d, const std::vector<double>& ends,
                       std::vector<double>& cp, std::vector<double>& iden)
{
    cp.assign((size_t)pmax * ny, 0.0);
    iden.assign((size_t)pmax * ny, 0.0);
    auto e = [&](int typ, int k, int j) { return ends[((size_t)typ * 4 + k) * ny + j]; };
    for (int j = 0; j < ny; ++j)
    {
        double cprev = 0;
        for (int p = 0; p < pmax; ++p)
        {
            const double lower = p > 0 ? -e(1, 1, j) : 0.0;
            const double diag  = d[j] - (p == 0 ? e(0, 3, j) : e(1, 3, j)) - e(1, 0, j);
            const double den   = diag - lower * cprev;
            const double c     = -e(1, 2, j) / den;
            cp[(size_t)p * ny + j]   = c;
            iden[(size_t)p * ny + j] = 1.0 / den;
            cprev                    = c;
        }
    }
}

template <typename T>
DevRect<T>::DevRect(int nx_, int ny_, double hx_, double hy_, const int* bc_, int sep_rows, bool with_transform)
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
    if (with_transform) tr.reset(new DevTransform<T>(kind, ny, true, true));
    singular  = !(dir_like(bc[0]) || dir_like(bc[1]) || dir_like(bc[2]) || dir_like(bc[3]));
    sing_from = ny - 1;
    build_chase_tables(x_diag(ny, hx, hy, bc[YNEG], bc[YPOS]), sep_rows);
}

template <typename T>
DevRect<T>::DevRect(int nx_, const std::vector<double>& d, int bc_xneg, int bc_xpos, bool singular_, int sing_from_)
    : nx(nx_), ny((int)d.size())
{
    bc[XNEG] = bc_xneg;
    bc[XPOS] = bc_xpos;
    bc[YNEG] = bc[YPOS] = BC_DIRICHLET;
    if (nx < 2 || ny < 1) throw Error(1, "each subdomain needs at least 2 cells per direction");
    const bool xp = bc_xneg == BC_PERIODIC && bc_xpos == BC_PERIODIC;
    if (!xp && (bc_xneg == BC_PERIODIC || bc_xpos == BC_PERIODIC || bc_xneg == BC_NULL || bc_xpos == BC_NULL))
        throw Error(1, "unsupported x boundary pair");
    singular  = singular_;
    sing_from = sing_from_;
    build_chase_tables(d, 0);
}

// Thomas tables of the nx x ny systems with diagonals d[j] (unit off-diagonals, the x boundary types of bc).
template <typename T> void DevRect<T>::build_chase_tables(const std::vector<double>& d, int sep_rows)
{
    const bool xp = bc[XNEG] == BC_PERIODIC && bc[XPOS] == BC_PERIODIC;
    periodic_x    = xp;
    std::vector<double> c;
    chase_table(nx, ny, d, !xp && bc[XNEG] == BC_NEUMANN, !xp && bc[XPOS] == BC_NEUMANN, c);
    ctab        = upload(convert<T>(c));
    end_neumann = !xp && bc[XPOS] == BC_NEUMANN;
    // the chunked kernels treat only the last wavenumber as singular
    chunked     = !xp && nx % kChunk == 0 && nx >= 2 * kChunk && (!singular || sing_from == ny - 1);
    if (chunked)
    {
        std::vector<double> pc, pg, ph, pe;
        partition_tables(ny, d, bc[XNEG] == BC_NEUMANN, pc, pg, ph, pe);
        cc    = upload(convert<T>(pc));
        cg    = upload(convert<T>(pg));
        chh   = upload(convert<T>(ph));
        cends = upload(convert<T>(pe));
        dsep  = upload(convert<T>(d));
        sep_pmax = std::max(sep_rows, nx / kChunk);
        std::vector<double> scp, sid;
        separator_factors(ny, sep_pmax, d, pe, scp, sid);
        sep_cp   = upload(convert<T>(scp));
        sep_iden = upload(convert<T>(sid));
    }
    if (periodic_x)
    {
        std::vector<double> a, b;
        periodic_tables(nx, ny, d, a, b);
        z1 = upload(convert<T>(a));
        z2 = upload(convert<T>(b));
    }
}

template <typename T> long long DevRect<T>::chase_scratch_elems(long long batch) const
{
    if (!chunked) return 0;
    const long long P = nx / kChunk;
    return batch * P * ny * 4;  // chunk end values (2), separator solution (1), separator scan slopes (1)
}

template <typename T> void DevRect<T>::chase(T* f, long long batch, T* scr, cudaStream_t s) const
{
    if (!chunked)
    {
        const long long nthreads = batch * ny;
        const int       block    = 128;
        k_chase<T><<<(unsigned)((nthreads + block - 1) / block), block, 0, s>>>(
            f, nx, ny, batch, ctab.as<T>(), z1.as<T>(), z2.as<T>(), periodic_x ? 1 : 0, singular ? 1 : 0, 0, sing_from);
        FPB_CHECK_LAUNCH();
        return;
    }
    const long long P    = nx / kChunk;
    T*              zend = scr;
    T*              bsep = zend + batch * P * ny * 2;
    T*              work = bsep + batch * P * ny;
    const int       skip = singular ? 1 : 0;
    const long long nl   = batch * P * ny;
    k_chase_local<T><<<(unsigned)((nl + 127) / 128), 128, 0, s>>>(f, nx, ny, batch, cc.as<T>(), cc.as<T>(), zend, skip);
    FPB_CHECK_LAUNCH();
    const long long nr = batch * ((ny + 31) / 32);  // CTAs: 32 wavenumbers of one field each
    k_chase_reduced<T><<<(unsigned)nr, 32 * kRedWarps, 0, s>>>(f, nx, ny, batch, cends.as<T>(), dsep.as<T>(),
                                                               end_neumann ? 1 : 0, zend, bsep, work,
                                                               sep_cp.as<T>(), sep_iden.as<T>(), skip);
    FPB_CHECK_LAUNCH();
    k_chase_correct<T><<<(unsigned)((nl + 255) / 256), 256, 0, s>>>(f, nx, ny, batch, cg.as<T>(), chh.as<T>(), bsep,
                                                                   skip);
    FPB_CHECK_LAUNCH();
    if (singular)
    {
        k_chase<T><<<(unsigned)((batch + 127) / 128), 128, 0, s>>>(f, nx, ny, batch, ctab.as<T>(), z1.as<T>(),
                                                                  z2.as<T>(), 0, 1, 1, ny - 1);
        FPB_CHECK_LAUNCH();
    }
}

template <typename T> void DevRect<T>::solve_mixed(T* f, long long batch, cudaStream_t s) const
{
    if (!std::is_same<T, double>::value) throw Error(1, "mixed-precision solve needs an FP64 plan");
    if (batch <= 0) return;
    if (!tr32) tr32.reset(new DevTransform<float>(tr->kind, ny, true, true));
    tr32->run_io<T>(f, f, batch * nx, false, s);
    const long long need = chase_scratch_elems(batch);
    if (need) scratch.ensure((size_t)need * sizeof(T));
    chase(f, batch, scratch.as<T>(), s);
    tr32->run_io<T>(f, f, batch * nx, true, s);
}

template <typename T> void DevRect<T>::solve(T* f, long long batch, cudaStream_t s) const
{
    if (batch <= 0) return;
    tr->run(f, f, batch * nx, false, s);
    const long long need = chase_scratch_elems(batch);
    if (need) scratch.ensure((size_t)need * sizeof(T));
    chase(f, batch, scratch.as<T>(), s);
    tr->run(f, f, batch * nx, true, s);
}

template <typename T> void DevRect<T>::chase_alone(T* f, long long batch, cudaStream_t s) const
{
    if (batch <= 0) return;
    const long long need = chase_scratch_elems(batch);
    if (need) scratch.ensure((size_t)need * sizeof(T));
    chase(f, batch, scratch.as<T>(), s);
}

template struct DevTransform<double>;
template struct DevTransform<float>;
template void DevTransform<float>::run_io<double>(const double*, double*, long long, bool, cudaStream_t) const;
template struct DevRect<double>;
template struct DevRect<float>;

}  // namespace fpb
