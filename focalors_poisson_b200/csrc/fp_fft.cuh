// Shared-memory complex FFT engine for one CTA.
//
// Layout: the whole length-M sequence lives in one shared-memory buffer of M complex values and is
// transformed in place by mixed-radix stages (radix 2, 3, 4, 5, 7, 8). Each butterfly reads and
// writes the same R slots, so one buffer suffices (no ping-pong), which is what lets an FP64
// transform of length ~13k fit in the 227 KB a CTA may own.
//
//  * DIF stages (natural order in)  -> spectrum in mixed-radix digit-reversed order
//  * DIT stages (digit-reversed in) -> spectrum in natural order
//
// A smooth length L is transformed by loading the input digit-reversed (a per-plan index table) and
// running the DIT stages. A length with a prime factor above 7 goes through Bluestein's chirp-z
// identity X_k = c_k * sum_n (x_n c_n) conj(c_{k-n}), c_n = exp(-i pi n^2 / L), restricted to a window:
// inputs n in [in0, in0+nin) (the others are zero) and outputs k in [out0, out0+nout) (the others are
// not needed). Then only the kernel lags -(nin-1) .. nout-1 occur and a cyclic convolution of smooth
// length M >= nin + nout - 1 is exact (2L-2 for the full window, whose two extreme lags share a value).
// Steps: DIF of (x c) placed from slot 0, pointwise product with the (digit-reversed, 1/M-scaled)
// transform of the kernel, conjugate, DIT, conjugate, times c_k; output k sits in slot k - out0.
//
// All twiddles, chirps and permutations are precomputed on the host in long double and read
// through the read-only cache.
#pragma once

#include "fp_common.cuh"

namespace fpb
{

constexpr int kFftMaxStages = 20;

struct FftStage
{
    int R;       // radix
    int S;       // span between butterfly legs
    int B;       // block size this stage works in (= R * S)
    int tw_off;  // twiddles for this stage: tw[tw_off + b] = exp(-2 pi i b / B); leg q uses its q-th power
};

struct FftDesc
{
    int      L;     // logical transform length
    int      M;     // executed length (L, or the Bluestein length)
    int      blue;  // 1: Bluestein
    int      in0, nin;    // Bluestein window: nonzero inputs [in0, in0+nin)
    int      out0, nout;  // and outputs kept [out0, out0+nout); (0, L, 0, L) for a direct transform
    int      eng;   // 0: the stage engine of this file; 1: the register engine (fp_fft16.cuh, M a power of 2);
                    // 2: the stage engine on a buffer in global memory (rows too long for shared memory)
    int      pad;   // shared-memory layout: element i in slot i + (i >> pad) (3 here, 4 for the register engine)
    int      lgM;   // log2 M (register engine)
    int      nst;
    FftStage st[kFftMaxStages];
};

// Shared-memory slot of FFT element i: one spare slot after every 8 elements. The butterflies of a
// power-of-two stage touch elements at strides 1, 8, 64, ... (times the radix); unpadded, 8 threads of a
// quarter warp (16-byte double2) or 16 of a half warp (8-byte float2) then hit one bank group, and the
// stages of 4096- and 8192-point FFTs ran at an eighth of shared-memory bandwidth. With the spare slot
// element i lands in bank group (i + i/8) mod 8 (mod 16 for float2), distinct across those threads.
__host__ __device__ __forceinline__ int fft_slot(int i) { return i + (i >> 3); }
// Slots an FFT buffer of executed length M occupies.
__host__ __device__ __forceinline__ int fft_buf_elems(int M) { return M + ((M + 7) >> 3); }

template <typename T2> struct FftTables
{
    const T2*   tw;      // stage twiddles
    const T2*   chirp;   // Bluestein: c_n, n < L
    const T2*   bhat;    // Bluestein: FFT_M(conj chirp kernel) / M, digit-reversed
    const int*  perm;    // direct: slot of input n for the DIT stages
    const int4* stages;  // (R, S, B, tw_off) per stage, read through the constant-like cache
};

// ---------------------------------------------------------------------------------------------
// Radix butterflies, forward sign exp(-2 pi i / R)
// ---------------------------------------------------------------------------------------------
template <typename T2> __device__ __forceinline__ void dft2(T2* x)
{
    T2 a = x[0], b = x[1];
    x[0] = a + b;
    x[1] = a - b;
}

template <typename T2> __device__ __forceinline__ void dft4(T2* x)
{
    T2 s0 = x[0] + x[2], s1 = x[0] - x[2], s2 = x[1] + x[3], s3 = mul_mi(x[1] - x[3]);
    x[0] = s0 + s2;
    x[2] = s0 - s2;
    x[1] = s1 + s3;
    x[3] = s1 - s3;
}

template <typename T2> __device__ __forceinline__ void dft8(T2* x)
{
    typedef decltype(T2::x) T;
    const T r = (T)0.70710678118654752440;
    T2 e[4] = {x[0], x[2], x[4], x[6]};
    T2 o[4] = {x[1], x[3], x[5], x[7]};
    dft4(e);
    dft4(o);
    // o_k *= w8^k : w8 = (1 - i)/sqrt2, w8^2 = -i, w8^3 = -(1 + i)/sqrt2
    T2 o1 = mk<T2>((o[1].x + o[1].y) * r, (o[1].y - o[1].x) * r);
    T2 o2 = mul_mi(o[2]);
    T2 o3 = mk<T2>((o[3].y - o[3].x) * r, -(o[3].x + o[3].y) * r);
    x[0] = e[0] + o[0];
    x[4] = e[0] - o[0];
    x[1] = e[1] + o1;
    x[5] = e[1] - o1;
    x[2] = e[2] + o2;
    x[6] = e[2] - o2;
    x[3] = e[3] + o3;
    x[7] = e[3] - o3;
}

template <typename T2> __device__ __forceinline__ void dft3(T2* x)
{
    typedef decltype(T2::x) T;
    const T s = (T)0.86602540378443864676;
    T2 t = x[1] + x[2], u = x[1] - x[2];
    T2 a = mk<T2>(x[0].x - (T)0.5 * t.x, x[0].y - (T)0.5 * t.y);
    T2 b = mk<T2>(s * u.y, -s * u.x);  // -i * s * u
    x[0] = x[0] + t;
    x[1] = a + b;
    x[2] = a - b;
}

template <typename T2> __device__ __forceinline__ void dft5(T2* x)
{
    typedef decltype(T2::x) T;
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    T2 t1 = x[1] + x[4], t2 = x[2] + x[3], t3 = x[1] - x[4], t4 = x[2] - x[3];
    T2 a1 = mk<T2>(x[0].x + c1 * t1.x + c2 * t2.x, x[0].y + c1 * t1.y + c2 * t2.y);
    T2 a2 = mk<T2>(x[0].x + c2 * t1.x + c1 * t2.x, x[0].y + c2 * t1.y + c1 * t2.y);
    T2 b1 = mk<T2>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    T2 b2 = mk<T2>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    x[0] = x[0] + t1 + t2;
    x[1] = a1 + mul_mi(b1);
    x[4] = a1 - mul_mi(b1);
    x[2] = a2 + mul_mi(b2);
    x[3] = a2 - mul_mi(b2);
}

template <typename T2> __device__ __forceinline__ void dft7(T2* x)
{
    typedef decltype(T2::x) T;
    const T C1 = (T)0.62348980185873353053, C2 = (T)-0.22252093395631440429, C3 = (T)-0.90096886790241912624;
    const T S1 = (T)0.78183148246802980871, S2 = (T)0.97492791218182360702, S3 = (T)0.43388373911755812048;
    T2 t1 = x[1] + x[6], t2 = x[2] + x[5], t3 = x[3] + x[4];
    T2 u1 = x[1] - x[6], u2 = x[2] - x[5], u3 = x[3] - x[4];
    T2 a1 = mk<T2>(x[0].x + C1 * t1.x + C2 * t2.x + C3 * t3.x, x[0].y + C1 * t1.y + C2 * t2.y + C3 * t3.y);
    T2 a2 = mk<T2>(x[0].x + C2 * t1.x + C3 * t2.x + C1 * t3.x, x[0].y + C2 * t1.y + C3 * t2.y + C1 * t3.y);
    T2 a3 = mk<T2>(x[0].x + C3 * t1.x + C1 * t2.x + C2 * t3.x, x[0].y + C3 * t1.y + C1 * t2.y + C2 * t3.y);
    // b_k = sum_m sin(2 pi m k / 7) u_m
    T2 b1 = mk<T2>(S1 * u1.x + S2 * u2.x + S3 * u3.x, S1 * u1.y + S2 * u2.y + S3 * u3.y);
    T2 b2 = mk<T2>(S2 * u1.x - S3 * u2.x - S1 * u3.x, S2 * u1.y - S3 * u2.y - S1 * u3.y);
    T2 b3 = mk<T2>(S3 * u1.x - S1 * u2.x + S2 * u3.x, S3 * u1.y - S1 * u2.y + S2 * u3.y);
    x[0] = x[0] + t1 + t2 + t3;
    x[1] = a1 + mul_mi(b1);
    x[6] = a1 - mul_mi(b1);
    x[2] = a2 + mul_mi(b2);
    x[5] = a2 - mul_mi(b2);
    x[3] = a3 + mul_mi(b3);
    x[4] = a3 - mul_mi(b3);
}

template <int R, typename T2> __device__ __forceinline__ void dft(T2* x)
{
    if constexpr (R == 2) dft2(x);
    else if constexpr (R == 3) dft3(x);
    else if constexpr (R == 4) dft4(x);
    else if constexpr (R == 5) dft5(x);
    else if constexpr (R == 7) dft7(x);
    else dft8(x);
}

// x[q] *= w^q for q = 1..R-1: odd powers w^(2j+1) = w^(2j-1) w^2 and even powers w^(2j) = w^(2j-2) w^2 as two
// interleaved chains, depth R/2 instead of R-2, three powers live (a few ulp either way).
template <int R, typename T2> __device__ __forceinline__ void rotate_legs(T2* x, T2 w1)
{
    x[1] = cmul(x[1], w1);
    if (R == 2) return;
    const T2 w2 = cmul(w1, w1);
    T2       wo = w1, we = w2;
    x[2]        = cmul(x[2], w2);
#pragma unroll
    for (int q = 3; q < R; ++q)
    {
        if (q & 1)
        {
            wo   = cmul(wo, w2);
            x[q] = cmul(x[q], wo);
        }
        else
        {
            we   = cmul(we, w2);
            x[q] = cmul(x[q], we);
        }
    }
}

// Leg q of butterfly b is rotated by w^q, w = exp(-2 pi i b / B): one table load per butterfly, the
// powers from it by rotate_legs.
// ld(k) supplies element k, sto(k, v) takes the result for element k: shared memory for an ordinary
// stage, the input pre-processing or the output post-processing for the fused first / last stages.
template <int R, bool DIT, typename T2, typename LD, typename ST>
__device__ __forceinline__ void stage_radix_io(const FftStage st, int nbf, const T2* __restrict__ tw, const LD& ld,
                                               const ST& sto)
{
    for (int t = threadIdx.x; t < nbf; t += blockDim.x)
    {
        const int blk  = t / st.S;
        const int b    = t - blk * st.S;
        const int base = blk * st.B + b;
        T2        x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = ld(base + q * st.S);
        const bool rot = b != 0;
        T2         w1  = rot ? __ldg(tw + st.tw_off + b) : mk<T2>(1, 0);
        if (DIT && rot) rotate_legs<R>(x, w1);
        dft<R>(x);
        if (!DIT && rot) rotate_legs<R>(x, w1);
#pragma unroll
        for (int q = 0; q < R; ++q) sto(base + q * st.S, x[q]);
    }
}

template <typename T2> struct SmemLd
{
    const T2* buf;
    __device__ __forceinline__ T2 operator()(int k) const { return buf[fft_slot(k)]; }
};
template <typename T2> struct SmemSt
{
    T2* buf;
    __device__ __forceinline__ void operator()(int k, T2 v) const { buf[fft_slot(k)] = v; }
};

__device__ __forceinline__ FftStage fft_stage(const int4* __restrict__ stages, int s)
{
    const int4 q = __ldg(stages + s);
    FftStage   st;
    st.R      = q.x;
    st.S      = q.y;
    st.B      = q.z;
    st.tw_off = q.w;
    return st;
}

template <bool DIT, typename T2, typename LD, typename ST>
__device__ __forceinline__ void stage_io(const FftStage st, int M, const T2* __restrict__ tw, const LD& ld, const ST& sto)
{
    const int nbf = M / st.R;
    switch (st.R)
    {
        case 2: stage_radix_io<2, DIT>(st, nbf, tw, ld, sto); break;
        case 3: stage_radix_io<3, DIT>(st, nbf, tw, ld, sto); break;
        case 4: stage_radix_io<4, DIT>(st, nbf, tw, ld, sto); break;
        case 5: stage_radix_io<5, DIT>(st, nbf, tw, ld, sto); break;
        case 7: stage_radix_io<7, DIT>(st, nbf, tw, ld, sto); break;
        default: stage_radix_io<8, DIT>(st, nbf, tw, ld, sto); break;
    }
}

// Runs stages [s0, s1) in place on buf, in DIF order (s0 first) or DIT order (s1 - 1 first), with a
// barrier after each.
template <bool DIT, typename T2>
__device__ void fft_stages(T2* buf, const FftDesc& d, const T2* __restrict__ tw, const int4* __restrict__ stages, int s0,
                           int s1)
{
    const SmemLd<T2> ld{buf};
    const SmemSt<T2> sto{buf};
    for (int i = s0; i < s1; ++i)
    {
        const int s = DIT ? s1 - 1 - (i - s0) : i;
        stage_io<DIT>(fft_stage(stages, s), d.M, tw, ld, sto);
        __syncthreads();
    }
}

// The last DIF stage, the product with the kernel transform and the first DIT stage in one pass: both
// stages have span 1 (no twiddles) and act on the same R consecutive elements, so the group stays in
// registers between them. Ends with a barrier.
template <int R, typename T2> __device__ __forceinline__ void stage_kernel_product_r(T2* buf, int M, const T2* __restrict__ bhat)
{
    for (int blk = threadIdx.x; blk < M / R; blk += blockDim.x)
    {
        T2 h[R], x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) h[q] = __ldg(bhat + blk * R + q);
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = buf[fft_slot(blk * R + q)];
        dft<R>(x);
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = cconj(cmul(x[q], h[q]));
        dft<R>(x);
#pragma unroll
        for (int q = 0; q < R; ++q) buf[fft_slot(blk * R + q)] = x[q];
    }
    __syncthreads();
}
template <typename T2> __device__ __forceinline__ void stage_kernel_product(T2* buf, int M, int R, const T2* __restrict__ bhat)
{
    switch (R)
    {
        case 2: stage_kernel_product_r<2>(buf, M, bhat); break;
        case 3: stage_kernel_product_r<3>(buf, M, bhat); break;
        case 4: stage_kernel_product_r<4>(buf, M, bhat); break;
        case 5: stage_kernel_product_r<5>(buf, M, bhat); break;
        case 7: stage_kernel_product_r<7>(buf, M, bhat); break;
        default: stage_kernel_product_r<8>(buf, M, bhat); break;
    }
}

// Slot in buf of input element i (i < L) of a direct transform before fft_execute: digit-reversed.
template <typename T2> __device__ __forceinline__ int fft_in_slot(const FftDesc& d, const FftTables<T2>& t, int i)
{
    return fft_slot(__ldg(t.perm + i));
}

// Elements one thread carries through a pass of an element-wise phase (pre- and post-processing): the
// pass issues the global and table loads of all of them before it stores any, so it waits for one
// memory latency per kFftBatch elements rather than one per element.
constexpr int kFftBatch = 4;

// Direct transform of the digit-reversed sequence in buf; on return buf holds the natural-order
// spectrum X_k, k < L (read with fft_out). Ends with a barrier.
template <typename T2> __device__ void fft_execute(T2* buf, const FftDesc& d, const FftTables<T2>& t)
{
    __syncthreads();
    fft_stages<true>(buf, d, t.tw, t.stages, 0, d.nst);
}

// Output store of the last Bluestein stage: X_{out0+k} = conj(y_k) c_{out0+k} for k in the window.
template <typename T2> struct PostChirpSt
{
    T2*                   buf;
    const T2* __restrict__ chirp;
    int                   out0, nout;
    __device__ __forceinline__ void operator()(int k, T2 v) const
    {
        if (k < nout) buf[fft_slot(k)] = cmul(cconj(v), __ldg(chirp + out0 + k));
    }
};

// Bluestein transform (d.blue, d.nst >= 2) of the input supplied by ld0: ld0(i) is the pre-chirped value
// of buffer position i (input element i + in0 times c_{i+in0}, zero outside the window). The input
// pre-processing runs inside the first DIF stage, the kernel product between the last DIF and first DIT
// stages, and the post-chirp inside the last DIT stage. On return buf holds X_k for k in the output
// window (fft_out). Starts and ends with a barrier.
template <typename T2, typename LD> __device__ void fft_execute_bluestein(T2* buf, const FftDesc& d, const FftTables<T2>& t, const LD& ld0)
{
    const int nst = d.nst;
    __syncthreads();
    stage_io<false>(fft_stage(t.stages, 0), d.M, t.tw, ld0, SmemSt<T2>{buf});
    __syncthreads();
    fft_stages<false>(buf, d, t.tw, t.stages, 1, nst - 1);
    stage_kernel_product(buf, d.M, fft_stage(t.stages, nst - 1).R, t.bhat);
    fft_stages<true>(buf, d, t.tw, t.stages, 1, nst - 1);
    stage_io<true>(fft_stage(t.stages, 0), d.M, t.tw, SmemLd<T2>{buf}, PostChirpSt<T2>{buf, t.chirp, d.out0, d.nout});
    __syncthreads();
}

// Slot of element i in the layout of plan d (either engine).
__host__ __device__ __forceinline__ int fft_slot_d(const FftDesc& d, int i) { return i + (i >> d.pad); }

// Spectrum value X_k after the transform, k in the output window (either engine).
template <typename T2> __device__ __forceinline__ T2 fft_out(const T2* buf, const FftDesc& d, int k)
{
    return buf[fft_slot_d(d, k - d.out0)];
}

// L - k for 0 < k <= L, and 0 for k = 0: the index of X_{-k}.
__device__ __forceinline__ int fft_mirror(int k, int L) { return k == 0 ? 0 : L - k; }

}  // namespace fpb
