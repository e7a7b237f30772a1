// y-direction transforms of the five boundary families (DD, NN, ND, DN, PP), forward and inverse,
// for a batch of contiguous rows. Each CTA owns one complex FFT of the family's real-DFT length L
// (2n+2, 2n, 2n+1, 2n+1, n) in shared memory. Two real sequences ride in one complex FFT:
//   * families that need one real DFT per row (DD, DN, forward NN / ND) pack two rows,
//   * families that need two real DFTs of the same row (inverse NN / ND, both PP directions) pack
//     the row's two sequences,
// and are separated afterwards with U_k = (Z_k + conj Z_{L-k})/2, V_k = (Z_k - conj Z_{L-k})/(2i).
// Pre- and post-processing restate the reference's per-family formulas
// (pe/poisson/poisson_fft2d.cpp:37-45, 92-133, 167-205, 232-262, 401-465) with tables computed by
// the same double expressions (fp_plan.cu), so results agree with the reference to FFT round-off.
#pragma once

#include "fp_fft.cuh"

namespace fpb
{

template <typename T> struct TransformArgs
{
    typedef typename Cplx<T>::type T2;
    const T*      in;
    T*            out;
    long long     rows;  // rows in the batch (fields * nx)
    int           n;     // row length (ny)
    FftDesc       fd;
    FftTables<T2> ft;
    const T*      ta;  // family table a (cos)
    const T*      tb;  // family table b (sin)
    T             s1, s2;
};

template <int KIND, int INV> struct FamilyTraits
{
    // true: one real DFT per row, two rows per FFT; false: two real DFTs of one row
    static constexpr bool kPairRows = (KIND == 0) || (KIND == 3) || (!INV && (KIND == 1 || KIND == 2));
};

template <typename T> __device__ __forceinline__ T alt_neg_even(int j) { return (j & 1) ? (T)1 : (T)-1; }
template <typename T> __device__ __forceinline__ T alt_pos_even(int j) { return (j & 1) ? (T)-1 : (T)1; }

template <typename T, int KIND, int INV>
__device__ __forceinline__ typename Cplx<T>::type build_input(const TransformArgs<T>& a, const T* fa, const T* fb, int i)
{
    typedef typename Cplx<T>::type T2;
    const int n = a.n;
    T         u = 0, v = 0;
    if (KIND == 0)  // DD: ex[j+1] = f_j (length 2n+2)
    {
        if (i >= 1 && i <= n)
        {
            u = fa[i - 1];
            v = fb ? fb[i - 1] : (T)0;
        }
    }
    else if (KIND == 1 && !INV)  // NN forward: ex[j+1] = (j even ? -1 : 1) f_j
    {
        if (i >= 1 && i <= n)
        {
            const T s = alt_neg_even<T>(i - 1);
            u         = s * fa[i - 1];
            v         = fb ? s * fb[i - 1] : (T)0;
        }
    }
    else if (KIND == 1 && INV)  // NN inverse: cos(..) p_j and sin(..) p_j
    {
        if (i >= 1 && i <= n)
        {
            const T p = fa[i - 1];
            u         = __ldg(a.ta + i - 1) * p;
            v         = __ldg(a.tb + i - 1) * p;
        }
    }
    else if ((KIND == 2 && !INV) || KIND == 3)  // ND forward, DN both: (j even ? -1 : 1) sqrt(4/(2n+1)) f_j
    {
        if (i >= 1 && i <= n)
        {
            const T s = alt_neg_even<T>(i - 1) * a.s1;
            u         = s * fa[i - 1];
            v         = fb ? s * fb[i - 1] : (T)0;
        }
    }
    else if (KIND == 2 && INV)  // ND inverse: sqrt(4/(2n+1)) sin(..) p_j and ... cos(..) p_j
    {
        if (i >= 1 && i <= n)
        {
            const T p = fa[i - 1];
            u         = (a.s1 * __ldg(a.tb + i - 1)) * p;
            v         = (a.s1 * __ldg(a.ta + i - 1)) * p;
        }
    }
    else if (KIND == 4 && !INV)  // PP forward: sin input [0, f_0..f_{n-2}], cos input alternating
    {
        if (i >= 1 && i <= n - 1)
        {
            const T f = fa[i - 1];
            u         = f;
            v         = alt_pos_even<T>(i - 1) * f;
        }
    }
    else  // PP inverse: even/odd cos parts summed into u, sin parts into v (poisson_fft2d.cpp:441-447)
    {
        const int h = n / 2;
        if (i < h) u += __ldg(a.ta + 2 * i) * fa[2 * i];
        if (i >= 1 && i <= h) u += __ldg(a.ta + 2 * i - 1) * fa[2 * i - 1];
        if (i >= 1 && i <= h) v += __ldg(a.tb + 2 * (h - i)) * fa[2 * (h - i)];
        if (i <= h - 1) v += __ldg(a.tb + 2 * (h - 1 - i) + 1) * fa[2 * (h - 1 - i) + 1];
    }
    return mk<T2>(u, v);
}

template <typename T, int KIND, int INV>
__global__ void __launch_bounds__(512) k_transform(const TransformArgs<T> a)
{
    typedef typename Cplx<T>::type T2;
    extern __shared__ __align__(16) unsigned char fp_smem_raw[];
    T2*          buf = reinterpret_cast<T2*>(fp_smem_raw);
    __shared__ T red[2][32];
    __shared__ T rowsc[2];

    constexpr bool kPair = FamilyTraits<KIND, INV>::kPairRows;
    const int      n     = a.n;
    const int      L     = a.fd.L;
    const long long r0   = kPair ? 2LL * blockIdx.x : (long long)blockIdx.x;
    if (r0 >= a.rows) return;
    const T* fa = a.in + r0 * n;
    const T* fb = (kPair && r0 + 1 < a.rows) ? fa + n : nullptr;
    T*       oa = a.out + r0 * n;
    T*       ob = (kPair && r0 + 1 < a.rows) ? oa + n : nullptr;

    // Row scalars needed after the FFT (read before any in-place write).
    if (threadIdx.x == 0)
    {
        if (KIND == 4 && !INV) rowsc[0] = fa[n - 1];  // PP forward: f(i, ny-1)
        if (KIND == 1 && INV) rowsc[0] = fa[n - 1];   // NN inverse: p_hat(i, ny-1)
    }
    if (KIND == 1 && !INV)  // NN forward mean slot: sum_j sqrt(1/n) f_j
    {
        T sa = 0, sb = 0;
        for (int j = threadIdx.x; j < n; j += blockDim.x)
        {
            sa += a.s2 * fa[j];
            if (fb) sb += a.s2 * fb[j];
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            sa += __shfl_down_sync(0xffffffffu, sa, o);
            sb += __shfl_down_sync(0xffffffffu, sb, o);
        }
        if ((threadIdx.x & 31) == 0)
        {
            red[0][threadIdx.x >> 5] = sa;
            red[1][threadIdx.x >> 5] = sb;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            T ta = 0, tb = 0;
            for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w)
            {
                ta += red[0][w];
                tb += red[1][w];
            }
            rowsc[0] = ta;
            rowsc[1] = tb;
        }
    }

    for (int i = threadIdx.x; i < a.fd.M; i += blockDim.x)
    {
        T2 z = (i < L) ? build_input<T, KIND, INV>(a, fa, fb, i) : mk<T2>(0, 0);
        buf[fft_in_slot(a.fd, a.ft, i)] = fft_in_value(a.fd, a.ft, i, z);
    }
    fft_execute(buf, a.fd, a.ft);

    const T half = (T)0.5;
    for (int j = threadIdx.x; j < n; j += blockDim.x)
    {
        const int k  = j + 1;
        const T2  Xk = fft_out(buf, a.fd, a.ft, k % L);
        const T2  Xm = fft_out(buf, a.fd, a.ft, (L - k) % L);
        // U = spectrum of the real part, V = spectrum of the imaginary part
        const T Ur = half * (Xk.x + Xm.x), Ui = half * (Xk.y - Xm.y);
        const T Vr = half * (Xk.y + Xm.y), Vi = -half * (Xk.x - Xm.x);
        if (KIND == 0)
        {
            oa[j] = -a.s1 * Ui;
            if (ob) ob[j] = -a.s1 * Vi;
        }
        else if (KIND == 1 && !INV)
        {
            if (j < n - 1)
            {
                const T c = __ldg(a.ta + j), s = __ldg(a.tb + j);
                oa[j] = a.s1 * (-c * Ui - s * Ur);
                if (ob) ob[j] = a.s1 * (-c * Vi - s * Vr);
            }
            else
            {
                oa[j] = rowsc[0];
                if (ob) ob[j] = rowsc[1];
            }
        }
        else if (KIND == 1 && INV)
        {
            oa[j] = alt_pos_even<T>(j) * a.s1 * Xk.y + (a.s1 + a.s2) * rowsc[0];
        }
        else if (KIND == 2 && !INV)
        {
            const T c = __ldg(a.ta + j), s = __ldg(a.tb + j);
            oa[j] = s * Ur - c * Ui;
            if (ob) ob[j] = s * Vr - c * Vi;
        }
        else if (KIND == 2 && INV)
        {
            oa[j] = alt_neg_even<T>(j) * Xk.x;
        }
        else if (KIND == 3)
        {
            oa[j] = alt_pos_even<T>(j) * Ui;
            if (ob) ob[j] = alt_pos_even<T>(j) * Vi;
        }
        else if (KIND == 4 && !INV)
        {
            const int h  = n / 2;
            const T   la = rowsc[0];
            T         ts = 0;
            if (j > 0)
            {
                const int ks = (j & 1) ? (h - (j - 1) / 2 - 1) : (h - j / 2);
                const T2  Sk = fft_out(buf, a.fd, a.ft, ks);
                const T2  Sm = fft_out(buf, a.fd, a.ft, (L - ks) % L);
                ts           = -(half * (Sk.y - Sm.y));
            }
            const int kc = (j & 1) ? (j + 1) / 2 : j / 2;
            const T2  Ck = fft_out(buf, a.fd, a.ft, kc);
            const T2  Cm = fft_out(buf, a.fd, a.ft, (L - kc) % L);
            const T   tc = la - half * (Ck.y + Cm.y);
            oa[j]        = a.s1 * (__ldg(a.ta + j) * ts + __ldg(a.tb + j) * tc);
        }
        else  // PP inverse
        {
            const int h  = n / 2;
            T         fc = 0, fs = 0;
            if (j < h)
            {
                fc = alt_neg_even<T>(j) * Ui;
                fs = Vr;
            }
            else if (j <= n - 2)
            {
                const int m  = n - 2 - j;
                const T2  Yk = fft_out(buf, a.fd, a.ft, m + 1);
                const T2  Ym = fft_out(buf, a.fd, a.ft, (L - m - 1) % L);
                fc           = -(alt_neg_even<T>(m) * (half * (Yk.y - Ym.y)));
                fs           = half * (Yk.y + Ym.y);
            }
            else
            {
                const T2 Y0 = fft_out(buf, a.fd, a.ft, 0);
                fs          = Y0.y;  // Re V_0 = Im Z_0
            }
            oa[j] = a.s1 * (fc + fs);
        }
    }
}

}  // namespace fpb
