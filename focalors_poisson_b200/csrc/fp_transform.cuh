// y-direction transforms of the five boundary families (DD, NN, ND, DN, PP), forward and inverse, for
// a batch of contiguous rows. Each CTA owns one complex FFT in shared memory. The transforms are the
// reference's PoissonFFT2D_* matrices (pe/poisson/poisson_fft2d.cpp:19-465), evaluated with the
// shortest complex FFT each family admits:
//
//   DD   DST-I of n = N+1 by the odd/even folding y_j = sin(pi j/n)(x_j + x_{n-j}) + (x_j - x_{n-j})/2:
//        X_{2k} = -Im Y_k, X_{2k+1} = X_{2k-1} + Re Y_k (a prefix sum), Y = DFT_n(y);  L = N+1
//   NN   DCT-II by Makhoul's reordering v = (f_0, f_2, ..., f_3, f_1), C_m = Re(e^{-i pi m/2N} V_m),
//        modes in the reference's order (mean last, others reversed and negated); the inverse is its
//        transpose, Re(DFT(e^{-i pi m/2N} a_m)) un-reordered;  L = N
//   ND   forward: the reference's length-(2N+1) real DFT; inverse: its transpose Re(DFT(beta p)) with
//        beta = sin + i cos of the reference's twiddles;  L = 2N+1
//   DN   the reference's length-(2N+1) real DFT (the family is its own transpose);  L = 2N+1
//   PP   the reference's two length-N real DFTs of one row packed in one complex FFT;  L = N
//
// Two real transforms share one complex FFT: for real-input families two rows ride as z = u + i v and
// separate as U_k = (Z_k + conj Z_{L-k})/2, V_k = (Z_k - conj Z_{L-k})/(2i); for real-output families
// (NN and ND inverses) two Hermitian-symmetrised rows ride as z = h_a + i h_b and come out as
// Re Z / Im Z. Every family except PP therefore costs half a complex FFT of length L per row.
// Family tables that the reference computes itself (ND, PP twiddles) are evaluated with its own double
// expressions (fp_plan.cu), so results agree with the reference to FFT round-off.
#pragma once

#include "fp_fft.cuh"
#include "fp_fft16.cuh"

namespace fpb
{

// T: arithmetic of the FFT; TIO: element type of the rows read and written (FP64 rows with an FP32 FFT
// is the reduced-precision transform of the iterative-refinement path).
// Everything a transform of one row length needs except the rows themselves.
template <typename T> struct XformArgs
{
    typedef typename Cplx<T>::type T2;
    int           n;  // row length (ny)
    FftDesc       fd;
    FftTables<T2> ft;
    const T*      ta;  // family table a (ND: cos, PP: cos, DD: sin(pi j/(N+1)) folding weights)
    const T*      tb;  // family table b (ND: sin, PP: sin)
    const T2*     tc;  // NN: exp(-i pi m / 2N)
    T             s1, s2;
    T2*           gbuf;     // eng 2: CTA b's FFT buffer (and DD scan arrays) at gbuf + b * gstride
    long long     gstride;
};

template <int KIND, int INV> struct FamilyTraits
{
    static constexpr bool kPairRows = (KIND != 4);
};

template <typename T> __device__ __forceinline__ T alt_neg_even(int j) { return (j & 1) ? (T)1 : (T)-1; }
template <typename T> __device__ __forceinline__ T alt_pos_even(int j) { return (j & 1) ? (T)-1 : (T)1; }

// Real input value u(i) of one row for the families whose FFT input is real.
template <typename T, int KIND, int INV, typename TA, typename TIO>
__device__ __forceinline__ T real_input(const TA& a, const TIO* f, int i)
{
    const int n = a.n;
    if (KIND == 0)  // DD folding, n+1 = L
    {
        if (i == 0) return (T)0;
        const T xj = (T)f[i - 1], xm = (T)f[n - i];  // x_j, x_{L-j}
        return __ldg(a.ta + i) * (xj + xm) + (T)0.5 * (xj - xm);
    }
    if (KIND == 1)  // NN forward: Makhoul reordering
        return (T)((2 * i < n) ? f[2 * i] : f[2 * n - 1 - 2 * i]);
    // ND forward, DN: ex[j+1] = (j even ? -1 : 1) sqrt(4/(2n+1)) f_j
    if (i >= 1 && i <= n) return (alt_neg_even<T>(i - 1) * a.s1) * (T)f[i - 1];
    return (T)0;
}

// Hermitian-symmetrised input h(i) of one row for the real-output families (NN / ND inverses).
template <typename T, int KIND, typename TA, typename TIO>
__device__ __forceinline__ typename Cplx<T>::type herm_input(const TA& a, const TIO* p, int i)
{
    typedef typename Cplx<T>::type T2;
    const int n = a.n;
    if (KIND == 1)  // NN inverse: c_m = w_m a_m, a_0 = sqrt(1/n) p_{n-1}, a_m = -sqrt(2/n) p_{n-1-m}
    {
        auto c = [&](int m) -> T2 {
            const T am = (m == 0) ? a.s2 * (T)p[n - 1] : -a.s1 * (T)p[n - 1 - m];
            const T2 w = a.tc[m];
            return mk<T2>(w.x * am, w.y * am);
        };
        const T2 c1 = c(i), c2 = c((n - i) % n);
        return mk<T2>((T)0.5 * (c1.x + c2.x), (T)0.5 * (c1.y - c2.y));
    }
    // ND inverse: g_t = (sin_b + i cos_b)_{t-1} p_{t-1} for 1 <= t <= n, zero elsewhere (L = 2n+1)
    if (i == 0) return mk<T2>(0, 0);
    if (i <= n)
    {
        const T p0 = (T)p[i - 1];
        return mk<T2>((T)0.5 * (__ldg(a.tb + i - 1) * p0), (T)0.5 * (__ldg(a.ta + i - 1) * p0));
    }
    const int t  = 2 * n + 1 - i;
    const T   p0 = (T)p[t - 1];
    return mk<T2>((T)0.5 * (__ldg(a.tb + t - 1) * p0), (T)-0.5 * (__ldg(a.ta + t - 1) * p0));
}

// PP: the row's two real sequences (poisson_fft2d.cpp:401-447).
template <typename T, int INV, typename TA, typename TIO>
__device__ __forceinline__ typename Cplx<T>::type pp_input(const TA& a, const TIO* f, int i)
{
    typedef typename Cplx<T>::type T2;
    const int n = a.n;
    T         u = 0, v = 0;
    if (!INV)  // sin input [0, f_0..f_{n-2}], cos input alternating from +f_0
    {
        if (i >= 1 && i <= n - 1)
        {
            u = (T)f[i - 1];
            v = alt_pos_even<T>(i - 1) * (T)f[i - 1];
        }
    }
    else  // even/odd cos parts summed into u, sin parts into v
    {
        const int h = n / 2;
        if (i < h) u += __ldg(a.ta + 2 * i) * (T)f[2 * i];
        if (i >= 1 && i <= h) u += __ldg(a.ta + 2 * i - 1) * (T)f[2 * i - 1];
        if (i >= 1 && i <= h) v += __ldg(a.tb + 2 * (h - i)) * (T)f[2 * (h - i)];
        if (i <= h - 1) v += __ldg(a.tb + 2 * (h - 1 - i) + 1) * (T)f[2 * (h - 1 - i) + 1];
    }
    return mk<T2>(u, v);
}

// Inclusive prefix sums of two arrays of length K in shared memory (one CTA).
template <typename T> __device__ void block_scan2(T* xa, T* xb, int K)
{
    __shared__ T wa[32], wb[32];
    const int    T_   = blockDim.x;
    const int    chunk = (K + T_ - 1) / T_;
    const int    lo = min(K, threadIdx.x * chunk), hi = min(K, lo + chunk);
    T            sa = 0, sb = 0;
    for (int k = lo; k < hi; ++k)
    {
        sa += xa[k];
        sb += xb[k];
    }
    // inclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T         ia = sa, ib = sb;
    for (int o = 1; o < 32; o <<= 1)
    {
        const T ya = __shfl_up_sync(0xffffffffu, ia, o), yb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o)
        {
            ia += ya;
            ib += yb;
        }
    }
    if (lane == 31)
    {
        wa[warp] = ia;
        wb[warp] = ib;
    }
    __syncthreads();
    if (warp == 0)
    {
        const int nw = (T_ + 31) / 32;
        T         va = lane < nw ? wa[lane] : (T)0, vb = lane < nw ? wb[lane] : (T)0;
        for (int o = 1; o < 32; o <<= 1)
        {
            const T ya = __shfl_up_sync(0xffffffffu, va, o), yb = __shfl_up_sync(0xffffffffu, vb, o);
            if (lane >= o)
            {
                va += ya;
                vb += yb;
            }
        }
        if (lane < nw)
        {
            wa[lane] = va;
            wb[lane] = vb;
        }
    }
    __syncthreads();
    T oa = ia - sa + (warp > 0 ? wa[warp - 1] : (T)0);
    T ob = ib - sb + (warp > 0 ? wb[warp - 1] : (T)0);
    for (int k = lo; k < hi; ++k)
    {
        oa += xa[k];
        ob += xb[k];
        xa[k] = oa;
        xb[k] = ob;
    }
    __syncthreads();
}

// Table values the output slot j of a family reads (NN forward: its post-twiddle; ND forward and PP
// forward: the reference's cos / sin pair), loaded in a batch before the slot's spectrum values.
template <typename T, int KIND, int INV>
__device__ __forceinline__ typename Cplx<T>::type out_table(const XformArgs<T>& a, int j)
{
    typedef typename Cplx<T>::type T2;
    const int n = a.n;
    if (KIND == 1 && !INV) return a.tc[(j < n - 1) ? n - 1 - j : 0];
    if ((KIND == 2 && !INV) || (KIND == 4 && !INV)) return mk<T2>(__ldg(a.ta + j), __ldg(a.tb + j));
    return mk<T2>(0, 0);
}

// Output values (row a, row b) of slot j for every family except DD, from the spectrum X in buf.
// tv: out_table(j); la: PP forward's f(i, ny-1).
template <typename T, int KIND, int INV>
__device__ __forceinline__ typename Cplx<T>::type out_value(const XformArgs<T>& a, const typename Cplx<T>::type* buf,
                                                          int j, typename Cplx<T>::type tv, T la)
{
    typedef typename Cplx<T>::type T2;
    const int n    = a.n;
    const int L    = a.fd.L;
    const T   half = (T)0.5;
    if (KIND == 1 && !INV)
    {
        // reference slot j holds mode m = n-1-j negated and scaled, the mean (m = 0) in slot n-1
        const int m  = (j < n - 1) ? n - 1 - j : 0;
        const T2  Zk = fft_out(buf, a.fd, m);
        const T2  Zm = fft_out(buf, a.fd, fft_mirror(m, L));
        const T2  w  = tv;  // (cos, -sin)(pi m / 2n)
        const T Ur = half * (Zk.x + Zm.x), Ui = half * (Zk.y - Zm.y);
        const T Vr = half * (Zk.y + Zm.y), Vi = -half * (Zk.x - Zm.x);
        const T Ca = w.x * Ur - w.y * Ui, Cb = w.x * Vr - w.y * Vi;  // Re(w V)
        const T sc = (j < n - 1) ? -a.s1 : a.s2;
        return mk<T2>(sc * Ca, sc * Cb);
    }
    else if (KIND == 1 && INV)
    {
        const int m = (j & 1) ? n - 1 - (j - 1) / 2 : j / 2;
        return fft_out(buf, a.fd, m);
    }
    else if (KIND == 2 && INV)
    {
        const T2 Z = fft_out(buf, a.fd, j + 1);
        const T  s = alt_neg_even<T>(j) * a.s1;
        return mk<T2>(s * Z.x, s * Z.y);
    }
    else if (KIND == 2 || KIND == 3)
    {
        const int k  = j + 1;
        const T2  Xk = fft_out(buf, a.fd, k);
        const T2  Xm = fft_out(buf, a.fd, fft_mirror(k, L));
        const T   Ur = half * (Xk.x + Xm.x), Ui = half * (Xk.y - Xm.y);
        const T   Vr = half * (Xk.y + Xm.y), Vi = -half * (Xk.x - Xm.x);
        if (KIND == 2)
        {
            const T c = tv.x, s = tv.y;
            return mk<T2>(s * Ur - c * Ui, s * Vr - c * Vi);
        }
        return mk<T2>(alt_pos_even<T>(j) * Ui, alt_pos_even<T>(j) * Vi);
    }
    else if (KIND == 4 && !INV)
    {
        const int h  = n / 2;
        T         ts = 0;
        if (j > 0)
        {
            const int ks = (j & 1) ? (h - (j - 1) / 2 - 1) : (h - j / 2);
            const T2  Sk = fft_out(buf, a.fd, ks);
            const T2  Sm = fft_out(buf, a.fd, fft_mirror(ks, L));
            ts           = -(half * (Sk.y - Sm.y));
        }
        const int kc = (j & 1) ? (j + 1) / 2 : j / 2;
        const T2  Ck = fft_out(buf, a.fd, kc);
        const T2  Cm = fft_out(buf, a.fd, fft_mirror(kc, L));
        const T   tc = la - half * (Ck.y + Cm.y);
        return mk<T2>(a.s1 * (tv.x * ts + tv.y * tc), (T)0);
    }
    else  // PP inverse
    {
        const int h  = n / 2;
        T         fc = 0, fs = 0;
        if (j < h)
        {
            const T2 Xk = fft_out(buf, a.fd, j + 1);
            const T2 Xm = fft_out(buf, a.fd, fft_mirror(j + 1, L));
            fc          = alt_neg_even<T>(j) * (half * (Xk.y - Xm.y));
            fs          = half * (Xk.y + Xm.y);
        }
        else if (j <= n - 2)
        {
            const int m  = n - 2 - j;
            const T2  Yk = fft_out(buf, a.fd, m + 1);
            const T2  Ym = fft_out(buf, a.fd, fft_mirror(m + 1, L));
            fc           = -(alt_neg_even<T>(m) * (half * (Yk.y - Ym.y)));
            fs           = half * (Yk.y + Ym.y);
        }
        else
        {
            fs = fft_out(buf, a.fd, 0).y;  // Re V_0 = Im Z_0
        }
        return mk<T2>(a.s1 * (fc + fs), (T)0);
    }
}

// Writes U output pairs v[u] to oa[idx[u]] (and ob[idx[u]] when ob), skipping idx < 0. ACC adds them
// to the values already there in FP64; those reads are issued together before the first store.
template <int U, bool ACC, typename TOUT, typename T2>
__device__ __forceinline__ void put_batch(TOUT* oa, TOUT* ob, const int* idx, const T2* v)
{
    double pa[U], pb[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
    {
        pa[u] = 0;
        pb[u] = 0;
        if (ACC && idx[u] >= 0)
        {
            pa[u] = (double)oa[idx[u]];
            if (ob) pb[u] = (double)ob[idx[u]];
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
    {
        if (idx[u] < 0) continue;
        if (ACC)
        {
            oa[idx[u]] = (TOUT)(pa[u] + (double)v[u].x);
            if (ob) ob[idx[u]] = (TOUT)(pb[u] + (double)v[u].y);
        }
        else
        {
            oa[idx[u]] = (TOUT)v[u].x;
            if (ob) ob[idx[u]] = (TOUT)v[u].y;
        }
    }
}

// Writes the DD output pairs of items k = k0 + u nt (u < U, k < K): out[2k] = ev[u] and, when 2k+1 < n,
// out[2k+1] = od[u], for row a (.x) and, when ob, row b (.y). vec: n is even and the rows are aligned to a
// pair, so each pair is one vector store (and one vector load for ACC). ACC adds to the values there in FP64.
template <typename TOUT> struct Pair;
template <> struct Pair<double>
{
    typedef double2 type;
};
template <> struct Pair<float>
{
    typedef float2 type;
};
template <int U, bool ACC, typename TOUT, typename T2>
__device__ __forceinline__ void put_pairs(TOUT* oa, TOUT* ob, int k0, int nt, int K, int n, bool vec, const T2* ev,
                                          const T2* od)
{
    typedef typename Pair<TOUT>::type P2;
    if (vec)
    {
        P2 pa[U], pb[U];
        if (ACC)
        {
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const int k = k0 + u * nt;
                if (k >= K) continue;
                pa[u] = reinterpret_cast<const P2*>(oa)[k];
                if (ob) pb[u] = reinterpret_cast<const P2*>(ob)[k];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int k = k0 + u * nt;
            if (k >= K) continue;
            P2 wa, wb;
            if (ACC)
            {
                wa.x = (TOUT)((double)pa[u].x + (double)ev[u].x);
                wa.y = (TOUT)((double)pa[u].y + (double)od[u].x);
                if (ob)
                {
                    wb.x = (TOUT)((double)pb[u].x + (double)ev[u].y);
                    wb.y = (TOUT)((double)pb[u].y + (double)od[u].y);
                }
            }
            else
            {
                wa.x = (TOUT)ev[u].x;
                wa.y = (TOUT)od[u].x;
                wb.x = (TOUT)ev[u].y;
                wb.y = (TOUT)od[u].y;
            }
            reinterpret_cast<P2*>(oa)[k] = wa;
            if (ob) reinterpret_cast<P2*>(ob)[k] = wb;
        }
        return;
    }
    int ie[U], io[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
    {
        const int k = k0 + u * nt;
        ie[u]       = k < K ? 2 * k : -1;
        io[u]       = (k < K && 2 * k + 1 < n) ? 2 * k + 1 : -1;
    }
    put_batch<U, ACC>(oa, ob, ie, ev);
    put_batch<U, ACC>(oa, ob, io, od);
}

// Shared memory of a register-engine plan: the exchange buffer, then the rotation table (M/16 entries),
// then the chirp tables (Bluestein plans); in elements of the complex type.
__host__ __device__ __forceinline__ int reg_tables_off(const FftDesc& d) { return reg_buf_elems(d.M); }
__host__ __device__ __forceinline__ int reg_smem_elems(const FftDesc& d)
{
    return reg_buf_elems(d.M) + (d.M >> 4) + (d.blue ? reg_chirp_entries(d.L) : 0);
}
// Register-engine kernels copy the plan's tables into shared memory once per CTA and plan.
template <typename T>
__device__ __forceinline__ void reg_tables_to_smem(const XformArgs<T>& a, typename Cplx<T>::type* buf)
{
    typedef typename Cplx<T>::type T2;
    T2* stw = buf + reg_tables_off(a.fd);
    reg_load_tables(a.fd, a.ft, stw, stw + (a.fd.M >> 4));
}

// One work item: rows fa (and fb, when has_b and the family pairs rows) of length a.n transformed into
// oa (ob). buf: the item's shared-memory FFT buffer; rowsc: two scratch values. ACC: out += result
// (FP64 accumulation of a correction) instead of out = result. ENG: the plan's FFT engine (0 stage
// engine, 1 register engine, whose tables the kernel has already put in shared memory after the buffer).
// Ends with the CTA synchronised. Every element-wise pass handles kFftBatch elements per thread at a
// time, loads first.
template <typename T, int KIND, int INV, typename TIN, typename TOUT, bool ACC, int ENG = 0, int MC = 0>
__device__ __forceinline__ void transform_rows(const XformArgs<T>& a, const TIN* fa, const TIN* fb, TOUT* oa, TOUT* ob,
                                               bool has_b, typename Cplx<T>::type* buf, T* rowsc)
{
    typedef typename Cplx<T>::type T2;
    constexpr bool kHerm = INV && (KIND == 1 || KIND == 2);  // real-output families
    constexpr int  U     = kFftBatch;
    const int      n     = a.n;
    const int      L     = a.fd.L;
    const int      M     = a.fd.M;
    const int      nt    = (int)blockDim.x;

    if (KIND == 4 && !INV && threadIdx.x == 0) rowsc[0] = (T)fa[n - 1];  // PP forward: f(i, ny-1)

    // FFT input (before any pre-chirp) of element e < L
    auto zval = [&](int e) -> T2 {
        if (KIND == 4) return pp_input<T, INV>(a, fa, e);
        if (kHerm)
        {
            const T2 ha = herm_input<T, KIND>(a, fa, e);
            const T2 hb = has_b ? herm_input<T, KIND>(a, fb, e) : mk<T2>(0, 0);
            return mk<T2>(ha.x - hb.y, ha.y + hb.x);  // h_a + i h_b
        }
        return mk<T2>(real_input<T, KIND, INV>(a, fa, e), has_b ? real_input<T, KIND, INV>(a, fb, e) : (T)0);
    };
    if constexpr (ENG == 1)
    {
        const T2* stw = buf + reg_tables_off(a.fd);
        reg_transform<MC>(buf, a.fd, a.ft, stw, stw + (M >> 4), zval);
    }
    else if (a.fd.blue)
    {
        auto ld0 = [&](int i) -> T2 {
            if (i >= a.fd.nin) return mk<T2>(0, 0);
            const int e = i + a.fd.in0;
            return cmul(zval(e), __ldg(a.ft.chirp + e));
        };
        fft_execute_bluestein(buf, a.fd, a.ft, ld0);
    }
    else
    {
        for (int i0 = threadIdx.x; i0 < M; i0 += U * nt)
        {
            T2  v[U];
            int sl[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const int i = i0 + u * nt;
                sl[u]       = (i < M) ? fft_in_slot(a.fd, a.ft, i) : -1;
                v[u]        = (i < M) ? zval(i) : mk<T2>(0, 0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (sl[u] >= 0) buf[sl[u]] = v[u];
        }
        fft_execute(buf, a.fd, a.ft);
    }

    const T half = (T)0.5;
    if (KIND == 0)
    {
        // DD: X_{2k} = -Im Y_k (k >= 1), X_{2k+1} = Re Y_0 / 2 + sum_{q=1..k} Re Y_q; out_m = s1 X_{m+1}, so
        // output pair k is out[2k] = s1 X_{2k+1} (k < K) and out[2k+1] = -s1 Im Y_{k+1} (2k+1 < n).
        const int K  = (n + 1) / 2;
        // scan arrays: the slots past element L-1 when the buffer has K of them, else past the buffer (and
        // the register engine's tables)
        const int lo = fft_slot_d(a.fd, L), hi = ENG == 1 ? reg_smem_elems(a.fd) : fft_buf_elems(M);
        T*        ca = reinterpret_cast<T*>(buf + ((hi - lo >= K) ? lo : hi));
        T*        cb = ca + K;
        for (int k = threadIdx.x; k < K; k += nt)
        {
            const T2 Zk = fft_out(buf, a.fd, k);
            const T2 Zm = fft_out(buf, a.fd, fft_mirror(k, L));
            const T  sc = (k == 0) ? (T)0.5 : (T)1;
            ca[k]       = sc * (half * (Zk.x + Zm.x));  // Re Y^a_k
            cb[k]       = sc * (half * (Zk.y + Zm.y));  // Re Y^b_k
        }
        __syncthreads();
        block_scan2(ca, cb, K);
        // Both outputs of a pair in one store where the rows allow it (n even, rows aligned to a pair).
        const bool vec = (n % 2 == 0) && (reinterpret_cast<uintptr_t>(oa) % (2 * sizeof(TOUT)) == 0);
        for (int k0 = threadIdx.x; k0 < K; k0 += U * nt)
        {
            T2 ev[U], od[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const int k = k0 + u * nt;
                ev[u]       = mk<T2>(0, 0);
                od[u]       = mk<T2>(0, 0);
                if (k >= K) continue;
                ev[u] = mk<T2>(a.s1 * ca[k], a.s1 * cb[k]);
                if (2 * k + 1 < n)
                {
                    const T2 Z1 = fft_out(buf, a.fd, k + 1);
                    const T2 Zm = fft_out(buf, a.fd, fft_mirror(k + 1, L));
                    od[u] = mk<T2>(a.s1 * (-(half * (Z1.y - Zm.y))), a.s1 * (half * (Z1.x - Zm.x)));  // -Im Y_{k+1}
                }
            }
            put_pairs<U, ACC>(oa, ob, k0, nt, K, n, vec, ev, od);
        }
        __syncthreads();
        return;
    }

    const T la = (KIND == 4 && !INV) ? rowsc[0] : (T)0;
    for (int j0 = threadIdx.x; j0 < n; j0 += U * nt)
    {
        T2 tv[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int j = j0 + u * nt;
            tv[u]       = (j < n) ? out_table<T, KIND, INV>(a, j) : mk<T2>(0, 0);
        }
        int idx[U];
        T2  v[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int j = j0 + u * nt;
            idx[u]      = (j < n) ? j : -1;
            v[u]        = (j < n) ? out_value<T, KIND, INV>(a, buf, j, tv[u], la) : mk<T2>(0, 0);
        }
        put_batch<U, ACC>(oa, ob, idx, v);
    }
    __syncthreads();
}

// Register caps. Stage engine: FP64 80, so that three CTAs of 256 threads fit per SM, as many as a
// 4096-point FP64 buffer allows. Register engine (16 complex values per thread, M/16 threads per CTA):
// FP64 128 (plans up to M = 8192, 512 threads, 64 K registers), FP32 64 (plans up to M = 16384, 1024
// threads).
template <int ENG, typename T> constexpr int xform_maxnreg()
{
    return ENG == 1 ? (sizeof(T) == 8 ? 128 : 64) : (sizeof(T) == 8 ? 80 : 64);  // ENG 2 as ENG 0
}

// Largest s with prefix[s] <= x (prefix ascending, prefix[0] = 0).
__device__ __forceinline__ int seg_of(const long long* __restrict__ prefix, int n, long long x)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A run of `rows` contiguous rows of one length transformed with plan `plan` (an index into the kernel's
// argument array: entries 2 plan and 2 plan + 1 are the forward and inverse arguments).
struct DstSeg
{
    const void* in;
    void*       out;
    int         rows, plan;
};

// The y-transform kernel of the library, for a single run of rows (the transform and rectangle entry
// points: segs == nullptr, the run passed by value in `one`) and for many runs of rows of several lengths in
// one persistent launch (the batched and composite solvers: a work list segs / prefix). One family and
// direction per launch; the per-row work is transform_rows.
// One work item = the rows one FFT carries (two for the pairing families) of one run; CTA b takes items
// b, b + gridDim.x, .... ACC: out (FP64) += result instead of out = result. DD and DN are their own
// transposes (the batched solver runs their inverse with INV = 0 and the forward arguments).
// PV (one plan for every run of the launch): the plan's arguments come by value in `pv`, in parameter space,
// which no store of the kernel can alias, so they are read as instruction operands instead of being reloaded
// into registers after the stores (measured on the 2048 x 2048 FP64 DD transform: 94 -> 87 us); otherwise
// the runs' plans are entries of the global array `plans` (entries 2 plan and 2 plan + 1 are the forward and
// inverse arguments of plan `plan`).
// Registers: uncapped, the stage engine's FP64 instances take 104-110, which allows only 2 CTAs of 256
// threads per SM, and at 80 (16 bytes of spill) three fit, as many as their shared memory allows (see
// xform_maxnreg).
// ENG 1 (register engine): every run of one launch has a plan of the same length M (M/16 threads per CTA);
// the CTA copies a plan's tables into shared memory when its items move to another plan. ENG 2 (rows whose
// FFT buffer does not fit in shared memory): the stage engine's code on a per-CTA buffer in global memory
// (XformArgs::gbuf, sized for the launch's grid), which the L2 keeps close.
template <typename T, int KIND, int INV, typename TIN, typename TOUT, bool ACC, int ENG, bool PV = false>
__global__ void __maxnreg__((xform_maxnreg<ENG, T>()))
    k_b_xform(const DstSeg* __restrict__ segs, const long long* __restrict__ prefix, int nseg, long long nitems,
              const XformArgs<T>* __restrict__ plans, const DstSeg one, const __grid_constant__ XformArgs<T> pv)
{
    typedef typename Cplx<T>::type T2;
    extern __shared__ __align__(16) unsigned char fp_smem_raw[];
    T2*            buf = reinterpret_cast<T2*>(fp_smem_raw);
    __shared__ T   rowsc[2];
    constexpr bool kPair  = FamilyTraits<KIND, INV>::kPairRows;
    int            loaded = -1;
    for (long long it = blockIdx.x; it < nitems; it += gridDim.x)
    {
        const int           s  = segs ? seg_of(prefix, nseg, it) : 0;
        const DstSeg        sg = segs ? segs[s] : one;
        const long long     i0 = segs ? prefix[s] : 0;
        const XformArgs<T>* Pp;
        if constexpr (PV) Pp = &pv;
        else Pp = plans + 2 * sg.plan + INV;
        const XformArgs<T>& P = *Pp;
        if constexpr (ENG == 2) buf = P.gbuf + blockIdx.x * P.gstride;
        if constexpr (ENG == 1)
        {
            const int pid = PV ? 0 : sg.plan;
            if (pid != loaded)
            {
                reg_tables_to_smem(P, buf);
                loaded = pid;
            }
        }
        const int       n     = P.n;
        const long long r0    = kPair ? 2 * (it - i0) : (it - i0);
        const bool      has_b = kPair && r0 + 1 < sg.rows;
        const TIN*      fa    = static_cast<const TIN*>(sg.in) + r0 * n;
        const TIN*      fb    = has_b ? fa + n : fa;
        TOUT*           oa    = static_cast<TOUT*>(sg.out) + r0 * n;
        TOUT*           ob    = has_b ? oa + n : nullptr;
        transform_rows<T, KIND, INV, TIN, TOUT, ACC, ENG>(P, fa, fb, oa, ob, has_b, buf, rowsc);
    }
}

// The register-engine length with a compile-time kernel (k_xform_rc); other lengths run k_b_xform.
constexpr int kXformStaticM = 4096;

// CTAs per SM the compile-time register-engine kernel is built for: FP64 2 (128 registers: 16 complex
// values per thread and no spill), FP32 3 (80 registers: measured on the 2048 x 2048 DD transform, 46 us
// against 47-48 us at 4 CTAs of 64 registers, which spill about 100 bytes, and 49 us at 2).
template <typename T> constexpr int xform_rc_ctas() { return sizeof(T) == 8 ? 2 : 3; }

// The register engine with one plan of compile-time length MC (M/16 = MC/16 threads per CTA) for every run
// of the launch: the plan's arguments by value in parameter space (see k_b_xform), its tables copied into
// shared memory once per CTA before the item loop, and launch bounds in place of a register cap, so that the
// compiler knows the CTA size. Runs: the work list segs / prefix, or the single run `one` (segs == nullptr).
// Measured on the 2048 x 2048 FP64 DD transform: 75 us, against 82-84 us for k_b_xform with the same plan by
// value (whose general item loop spilled 48 bytes per thread at its register cap).
template <typename T, int KIND, int INV, typename TIN, typename TOUT, bool ACC, int MC>
__global__ void __launch_bounds__(MC / 16, xform_rc_ctas<T>())
    k_xform_rc(const DstSeg* __restrict__ segs, const long long* __restrict__ prefix, int nseg, long long nitems,
               const DstSeg one, const __grid_constant__ XformArgs<T> P)
{
    typedef typename Cplx<T>::type T2;
    extern __shared__ __align__(16) unsigned char fp_smem_raw[];
    T2*            buf = reinterpret_cast<T2*>(fp_smem_raw);
    __shared__ T   rowsc[2];
    constexpr bool kPair = FamilyTraits<KIND, INV>::kPairRows;
    reg_tables_to_smem(P, buf);
    const int n = P.n;
    for (long long it = blockIdx.x; it < nitems; it += gridDim.x)
    {
        const int       s     = segs ? seg_of(prefix, nseg, it) : 0;
        const DstSeg    sg    = segs ? segs[s] : one;
        const long long i0    = segs ? prefix[s] : 0;
        const long long r0    = kPair ? 2 * (it - i0) : (it - i0);
        const bool      has_b = kPair && r0 + 1 < sg.rows;
        // The rows of this CTA's next item into L2 (one 128-byte line per thread and step), so that its load
        // phase waits for L2 rather than HBM.
        const long long nx = it + gridDim.x;
        if (nx < nitems)
        {
            const int       s2  = segs ? seg_of(prefix, nseg, nx) : 0;
            const DstSeg    sg2 = segs ? segs[s2] : one;
            const long long q0  = kPair ? 2 * (nx - (segs ? prefix[s2] : 0)) : (nx - (segs ? prefix[s2] : 0));
            const long long nr  = (kPair && q0 + 1 < sg2.rows) ? 2 : 1;
            const char*     pb  = reinterpret_cast<const char*>(static_cast<const TIN*>(sg2.in) + q0 * n);
            const long long nb  = nr * n * (long long)sizeof(TIN);
            for (long long o = (long long)threadIdx.x * 128; o < nb; o += (long long)blockDim.x * 128)
                asm volatile("prefetch.L2 [%0];" ::"l"(pb + o));
        }
        const TIN*      fa    = static_cast<const TIN*>(sg.in) + r0 * n;
        const TIN*      fb    = has_b ? fa + n : fa;
        TOUT*           oa    = static_cast<TOUT*>(sg.out) + r0 * n;
        TOUT*           ob    = has_b ? oa + n : nullptr;
        transform_rows<T, KIND, INV, TIN, TOUT, ACC, 1, MC>(P, fa, fb, oa, ob, has_b, buf, rowsc);
    }
}

}  // namespace fpb
