// Register-resident Stockham FFT engine for power-of-two lengths M >= 512 (one FFT per CTA).
//
// Thread t of T = M/16 holds the 16 elements t + T q (q = 0..15) of the sequence in registers: the
// "column" layout. The transform is the radix-R Stockham autosort: pass p with span Ns (the product of
// the radices before it) takes butterflies j = 0..M/R-1 on the elements j + r M/R (r < R), rotates leg r
// by w^(r (j mod Ns)), w = exp(-2 pi i / (Ns R)), runs the R-point DFT and sends leg r to element
// (j / Ns) Ns R + (j mod Ns) + r Ns. Thread t owns the butterflies j = t + b T (b < 16/R), whose legs are
// exactly its own column registers q = b + r 16/R, so every pass reads the column layout; between passes
// the results go through shared memory once (write at the destination index, barrier, read the column,
// barrier). In the last pass (Ns R = M) the destination is the column itself, so the natural-order
// spectrum ends in the registers with no exchange.
//
// Passes: a radix 2^(log2 M mod 4) pass first (span 1, no rotation) when log2 M is not a multiple of 4,
// then radix-16 passes (each a 4 x 4 split with constant internal rotations). M = 4096 takes three passes
// and two exchanges, where a stage-per-sweep radix-8 engine takes four sweeps of shared memory.
//
// Bluestein (a length L whose FFT is computed as a cyclic convolution of length M, see fp_fft.cuh for the
// windowed form): the pre-chirped input is loaded from the rows straight into the column registers, the
// forward FFT ends with the spectrum in registers, the product with the kernel transform (natural order,
// read from global memory in the column layout, coalesced) and the conjugation happen in registers, and
// the second FFT starts from them: the kernel product costs no shared-memory sweep at all. The chirp
// c_e = exp(-i pi e^2 / L), e < L, and the pass rotations exp(-2 pi i m / M), m < M/16, are tables that
// each CTA copies from global memory into shared memory once.
//
// Shared memory: element i lives in slot i + i/16 (the radix-16 destinations j*16 + r of the first pass
// then fall in distinct bank groups across a quarter warp for 16-byte elements and a half warp for
// 8-byte ones).
#pragma once

#include "fp_fft.cuh"

namespace fpb
{

constexpr int kRegE    = 16;   // elements per thread
constexpr int kRegPad  = 4;    // slot(i) = i + (i >> kRegPad)
constexpr int kRegMinM = 512;  // at least one warp per FFT

__host__ __device__ __forceinline__ int reg_slot(int i) { return i + (i >> kRegPad); }
__host__ __device__ __forceinline__ int reg_buf_elems(int M) { return M + (M >> kRegPad); }
// Entries of the chirp table for length L: c_e, e < L.
__host__ __device__ __forceinline__ int reg_chirp_entries(int L) { return L; }

// v * exp(-2 pi i m / 16) for a compile-time m in 0..15.
template <int m, typename T2> __device__ __forceinline__ T2 w16mul(T2 v)
{
    typedef decltype(T2::x) T;
    constexpr int k = m & 15;
    const T       c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, r = (T)0.70710678118654752440;
    if constexpr (k == 0) return v;
    else if constexpr (k == 4) return mk<T2>(v.y, -v.x);
    else if constexpr (k == 8) return mk<T2>(-v.x, -v.y);
    else if constexpr (k == 12) return mk<T2>(-v.y, v.x);
    else
    {
        // exp(-2 pi i k / 16) = (cos, -sin)
        constexpr int q = k & 3, h = k >> 2;  // k = 4 h + q, q in 1..3
        T cs, sn;
        if constexpr (q == 1) { cs = c1; sn = s1; }
        else if constexpr (q == 2) { cs = r; sn = r; }
        else { cs = s1; sn = c1; }
        // rotate by exp(-2 pi i q / 16), then by (-i)^h
        T2 w = mk<T2>(v.x * cs + v.y * sn, v.y * cs - v.x * sn);
        if constexpr (h == 1) return mk<T2>(w.y, -w.x);
        else if constexpr (h == 2) return mk<T2>(-w.x, -w.y);
        else if constexpr (h == 3) return mk<T2>(-w.y, w.x);
        else return w;
    }
}

template <int n2, int k1, typename T2> __device__ __forceinline__ T2 w16_at(T2 v) { return w16mul<n2 * k1>(v); }

// 16-point DFT, natural order in and out, as 4 x 4: x[4 n1 + n2] -> 4-point DFTs over n1, rotation by
// w16^(n2 k1), 4-point DFTs over n2, X[k1 + 4 k2].
template <typename T2> __device__ __forceinline__ void dft16(T2* x)
{
    T2 a[4][4];  // a[n2][k1]
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2)
    {
        T2 u[4] = {x[n2], x[4 + n2], x[8 + n2], x[12 + n2]};
        dft4(u);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = u[k1];
    }
    a[1][1] = w16_at<1, 1>(a[1][1]);
    a[1][2] = w16_at<1, 2>(a[1][2]);
    a[1][3] = w16_at<1, 3>(a[1][3]);
    a[2][1] = w16_at<2, 1>(a[2][1]);
    a[2][2] = w16_at<2, 2>(a[2][2]);
    a[2][3] = w16_at<2, 3>(a[2][3]);
    a[3][1] = w16_at<3, 1>(a[3][1]);
    a[3][2] = w16_at<3, 2>(a[3][2]);
    a[3][3] = w16_at<3, 3>(a[3][3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
    {
        T2 u[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
        dft4(u);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) x[k1 + 4 * k2] = u[k2];
    }
}

template <int R, typename T2> __device__ __forceinline__ void reg_dft(T2* x)
{
    if constexpr (R == 16) dft16(x);
    else if constexpr (R == 8) dft8(x);
    else if constexpr (R == 4) dft4(x);
    else dft2(x);
}

// One Stockham pass of radix R and span Ns on the column registers (see the file comment). tw: the
// shared-memory table exp(-2 pi i m / M), m < M/16; the rotation base of butterfly j is entry
// (j mod Ns) * M / (16 Ns) (radix-16 passes; the radix < 16 pass has span 1 and no rotation).
template <int R, typename T2>
__device__ __forceinline__ void reg_pass(T2 (&v)[kRegE], int t, int T, int Ns, int tws, const T2* __restrict__ tw)
{
    constexpr int B = kRegE / R;
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        T2 x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = v[b + r * B];
        if (Ns > 1)
        {
            const int k = (t + b * T) & (Ns - 1);
            if (k) rotate_legs<R>(x, tw[k * tws]);
        }
        reg_dft<R>(x);
#pragma unroll
        for (int r = 0; r < R; ++r) v[b + r * B] = x[r];
    }
}

// After a pass that is not the last: legs to their destinations in shared memory, then the column back.
template <int R, typename T2> __device__ __forceinline__ void reg_exchange(T2 (&v)[kRegE], T2* buf, int t, int T, int Ns)
{
    constexpr int B = kRegE / R;
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j    = t + b * T;
        const int base = (j & ~(Ns - 1)) * R + (j & (Ns - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) buf[reg_slot(base + r * Ns)] = v[b + r * B];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kRegE; ++q) v[q] = buf[reg_slot(t + T * q)];
    __syncthreads();
}

// Forward FFT (exp(-2 pi i ...)) of length M = 2^lgM held in the column registers; natural order in and
// out. buf: the CTA's shared-memory exchange buffer (reg_buf_elems(M) slots); no thread may still be
// reading it from an earlier use (callers end every use with a barrier).
template <typename T2>
__device__ __forceinline__ void reg_fft(T2 (&v)[kRegE], T2* buf, int M, int lgM, const T2* __restrict__ tw)
{
    const int t  = threadIdx.x, T = M >> 4;
    int       Ns = 1;
    switch (lgM & 3)
    {
        case 1: reg_pass<2>(v, t, T, 1, 0, tw); reg_exchange<2>(v, buf, t, T, 1); Ns = 2; break;
        case 2: reg_pass<4>(v, t, T, 1, 0, tw); reg_exchange<4>(v, buf, t, T, 1); Ns = 4; break;
        case 3: reg_pass<8>(v, t, T, 1, 0, tw); reg_exchange<8>(v, buf, t, T, 1); Ns = 8; break;
        default: break;
    }
    while (Ns < M)
    {
        reg_pass<16>(v, t, T, Ns, M / (16 * Ns), tw);
        if (Ns * 16 < M) reg_exchange<16>(v, buf, t, T, Ns);
        Ns *= 16;
    }
}

// The same passes with the length M known at compile time (k_xform_rc instantiates M = 4096: the Bluestein
// length of DST-I rows of 1025..2048 and the direct length of NN / PP rows of 4096). Spans, rotation strides
// and every shared-memory slot become constants or constant offsets from one per-thread base, which takes the
// slot arithmetic out of the exchanges and frees the registers it held (2048 x 2048 FP64 DD transform, plan
// already passed by value: 87 -> 83 us).
template <int R, int Ns, int M, typename T2>
__device__ __forceinline__ void reg_pass_c(T2 (&v)[kRegE], int t, const T2* __restrict__ tw)
{
    constexpr int B = kRegE / R, T = M / 16, tws = Ns > 1 ? M / (16 * Ns) : 0;
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        T2 x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = v[b + r * B];
        if constexpr (Ns > 1)
        {
            const int k = (t + b * T) & (Ns - 1);
            if (k) rotate_legs<R>(x, tw[k * tws]);
        }
        reg_dft<R>(x);
#pragma unroll
        for (int r = 0; r < R; ++r) v[b + r * B] = x[r];
    }
}

template <int R, int Ns, int M, typename T2> __device__ __forceinline__ void reg_exchange_c(T2 (&v)[kRegE], T2* buf, int t)
{
    constexpr int B = kRegE / R, T = M / 16;
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j    = t + b * T;
        const int base = (j & ~(Ns - 1)) * R + (j & (Ns - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) buf[reg_slot(base + r * Ns)] = v[b + r * B];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kRegE; ++q) v[q] = buf[reg_slot(t + T * q)];
    __syncthreads();
}

// Radix-16 passes of span Ns, Ns * 16, ... up to M (the last one without an exchange).
template <int Ns, int M, typename T2>
__device__ __forceinline__ void reg_passes16_c(T2 (&v)[kRegE], T2* buf, int t, const T2* __restrict__ tw)
{
    reg_pass_c<16, Ns, M>(v, t, tw);
    if constexpr (Ns * 16 < M)
    {
        reg_exchange_c<16, Ns, M>(v, buf, t);
        reg_passes16_c<Ns * 16, M>(v, buf, t, tw);
    }
}

template <int M, typename T2> __device__ __forceinline__ void reg_fft_c(T2 (&v)[kRegE], T2* buf, const T2* __restrict__ tw)
{
    static_assert(M >= kRegMinM && (M & (M - 1)) == 0, "register engine: a power of two >= 512");
    const int     t   = threadIdx.x;
    constexpr int lg  = __builtin_ctz(M);
    constexpr int r0  = 1 << (lg & 3);  // radix of the first pass when log2 M is not a multiple of 4
    if constexpr (r0 > 1)
    {
        reg_pass_c<r0, 1, M>(v, t, tw);
        reg_exchange_c<r0, 1, M>(v, buf, t);
        reg_passes16_c<r0, M>(v, buf, t, tw);
    }
    else
        reg_passes16_c<1, M>(v, buf, t, tw);
}

// reg_fft with a compile-time length MC, or the run-time d.M when MC is 0.
template <int MC, typename T2>
__device__ __forceinline__ void reg_fft_m(T2 (&v)[kRegE], T2* buf, const FftDesc& d, const T2* __restrict__ tw)
{
    if constexpr (MC > 0) reg_fft_c<MC>(v, buf, tw);
    else reg_fft(v, buf, d.M, d.lgM, tw);
}

// c_e = exp(-i pi e^2 / L) from the chirp table in shared memory (0 <= e < L).
template <typename T2> __device__ __forceinline__ T2 reg_chirp(const T2* __restrict__ ch, int e, int) { return ch[e]; }

// Copies the rotation table (M/16 entries) and, for Bluestein plans, the chirp table into shared memory.
// Ends with a barrier.
template <typename T2>
__device__ __forceinline__ void reg_load_tables(const FftDesc& d, const FftTables<T2>& ft, T2* stw, T2* sch)
{
    for (int i = threadIdx.x; i < (d.M >> 4); i += blockDim.x) stw[i] = __ldg(ft.tw + i);
    if (d.blue)
        for (int i = threadIdx.x; i < reg_chirp_entries(d.L); i += blockDim.x) sch[i] = __ldg(ft.chirp + i);
    __syncthreads();
}

// The complex DFT of length d.L of the input zval(e) (e < L) on the register engine. On return the spectrum
// values X_k of the output window sit in buf at reg_slot(k - d.out0) (fft_out), followed by a barrier.
// d.blue: Bluestein with the windowed kernel transform ft.bhat (natural order, scaled 1/M); else L = M.
// MC: the length M at compile time (d.M == MC), or 0.
template <int MC = 0, typename T2, typename ZV>
__device__ __forceinline__ void reg_transform(T2* buf, const FftDesc& d, const FftTables<T2>& ft,
                                              const T2* __restrict__ stw, const T2* __restrict__ sch, const ZV& zval)
{
    T2        v[kRegE];
    const int t = threadIdx.x, M = MC > 0 ? MC : d.M, T = M >> 4, L = d.L;
    if (d.blue)
    {
#pragma unroll
        for (int q = 0; q < kRegE; ++q)
        {
            const int i = t + T * q;
            v[q]        = mk<T2>(0, 0);
            if (i < d.nin)
            {
                const int e = i + d.in0;
                v[q]        = cmul(zval(e), reg_chirp(sch, e, L));
            }
        }
        reg_fft_m<MC>(v, buf, d, stw);
#pragma unroll
        for (int q = 0; q < kRegE; ++q) v[q] = cconj(cmul(v[q], __ldg(ft.bhat + t + T * q)));
        reg_fft_m<MC>(v, buf, d, stw);
#pragma unroll
        for (int q = 0; q < kRegE; ++q)
        {
            const int p = t + T * q;
            if (p < d.nout) buf[reg_slot(p)] = cmul(cconj(v[q]), reg_chirp(sch, d.out0 + p, L));
        }
    }
    else
    {
#pragma unroll
        for (int q = 0; q < kRegE; ++q) v[q] = zval(t + T * q);
        reg_fft_m<MC>(v, buf, d, stw);
#pragma unroll
        for (int q = 0; q < kRegE; ++q) buf[reg_slot(t + T * q)] = v[q];
    }
    __syncthreads();
}

}  // namespace fpb
