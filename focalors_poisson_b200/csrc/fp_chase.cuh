// Batched tridiagonal "chasing" along x, one system per (field, wavenumber), restating
// ChasingMethod2D::chasing (pe/poisson/chasing_method2d.cpp:44-89) and the solvers of
// pe/poisson/chasing_method_base.cpp: Thomas with unit off-diagonals (:24-52), the singular
// recursion x0 = 0 (:146-154), Sherman-Morrison for periodic x (:178-197) and the singular periodic
// formula (:267-279).
//
// No transpose: after the y-transform the field is still row-major (x, wavenumber), so thread j walks
// column j and a warp reads 32 consecutive wavenumbers of one row per step (coalesced).
//
// ctab holds, per wavenumber j and row i: c_i = 1/(d_j - c_{i-1}) for i < nx-1 with
// c_0 = 1/(d_j [+1 if x- Neumann]) and, in row nx-1, 1/(d_j [+1 if x+ Neumann] - c_{nx-2}), so that
// y_0 = f_0 c_0, y_i = (f_i - y_{i-1}) c_i, x_{n-1} = y_{n-1}, x_i = y_i - c_i x_{i+1}.
#pragma once

#include "fp_common.cuh"

namespace fpb
{

// only_last: one thread per field, handling just the last wavenumber (the singular one), for use next
// to the chunked kernels below. With `singular`, the wavenumbers j >= sing_from take the singular
// recursions: the last one (sing_from = ny - 1) in 2D and in 3D without periodic x; in 3D with periodic x
// the reference applies the singular periodic formula to every y-mode of the last z-mode
// (pe/poisson/chasing_method3d.cpp:55-76), sing_from = (nz - 1) ny in the combined mode index.
template <typename T>
__global__ void k_chase(T* __restrict__ f, int nx, int ny, long long batch, const T* __restrict__ ctab,
                        const T* __restrict__ z1, const T* __restrict__ z2, int periodic, int singular,
                        int only_last, int sing_from)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (only_last ? batch : batch * ny)) return;
    const int       j   = only_last ? ny - 1 : (int)(t % ny);
    const long long b   = only_last ? t : t / ny;
    T*              col = f + b * (long long)nx * ny + j;
    const long long s   = ny;

    if (singular && j >= sing_from)
    {
        if (!periodic)
        {
            // x0 = 0, x1 = f0, x_i = f_{i-1} - x_{i-2} + 2 x_{i-1}
            T fprev = col[0];
            col[0]  = 0;
            T xm2 = 0, xm1 = (T)0 + fprev;
            if (nx > 1)
            {
                fprev  = col[s];
                col[s] = xm1;
            }
            for (int i = 2; i < nx; ++i)
            {
                const T fi = col[i * s];
                const T x  = fprev - xm2 + (T)2 * xm1;
                col[i * s] = x;
                xm2        = xm1;
                xm1        = x;
                fprev      = fi;
            }
        }
        else
        {
            // x0 = 0, x1 = f0/n - sum_{i=1}^{n-2} (n-1-i) f_i / n, then the same recursion
            const int n  = nx;
            T         x1 = col[0] / (T)n;
            for (int i = 1; i < n - 1; ++i) x1 = x1 - (T)(n - 1 - i) * col[i * s] / (T)n;
            T fprev = col[0];
            col[0]  = 0;
            T xm2 = 0, xm1 = x1;
            if (n > 1)
            {
                fprev  = col[s];
                col[s] = xm1;
            }
            for (int i = 2; i < n; ++i)
            {
                const T fi = col[i * s];
                const T x  = fprev - xm2 + (T)2 * xm1;
                col[i * s] = x;
                xm2        = xm1;
                xm1        = x;
                fprev      = fi;
            }
        }
        return;
    }

    // Thomas forward sweep (y overwrites f) and back substitution (x overwrites y).
    const T* cj = ctab + j;
    T        y  = col[0] * __ldg(cj);
    col[0]      = y;
    for (int i = 1; i < nx; ++i)
    {
        y          = (col[i * s] - y) * __ldg(cj + i * s);
        col[i * s] = y;
    }
    T x = y;
    for (int i = nx - 2; i >= 0; --i)
    {
        x          = col[i * s] - __ldg(cj + i * s) * x;
        col[i * s] = x;
    }
    if (!periodic) return;

    // Sherman-Morrison correction with the two precomputed special solutions.
    const T* a  = z1 + j;
    const T* bb = z2 + j;
    const T  y0 = col[0], yl = col[(nx - 1) * s];
    const T  a0 = __ldg(a), al = __ldg(a + (nx - 1) * s), b0 = __ldg(bb), bl = __ldg(bb + (nx - 1) * s);
    const T  g2 = (yl / ((T)1 + al) - y0 / a0) / (bl / ((T)1 + al) - ((T)1 + b0) / a0);
    const T  g1 = y0 / a0 - g2 * (((T)1 + b0) / a0);
    for (int i = 0; i < nx; ++i) col[i * s] = col[i * s] - g1 * __ldg(a + i * s) - g2 * __ldg(bb + i * s);
}

}  // namespace fpb

namespace fpb
{

// ---------------------------------------------------------------------------------------------
// Chunked ("partition") form of the same Thomas solve for the standard (Dirichlet / Neumann ends)
// systems, used when nx is a multiple of kChunk. Rows are cut into P = nx / kChunk chunks; the last
// row of every chunk is a separator. The kChunk-1 interior rows of chunk p satisfy
//   x_int = z_p - B_{p-1} g - B_p h,   z_p = T^-1 f_int, g = T^-1 e_first, h = T^-1 e_last,
// with B_p the separator values; the separator equations then form a tridiagonal system of size P:
//   -g_last B_{p-1} + (d_sep - h_last - g'_first) B_p - h'_first B_{p+1} = f_sep - z_p,last - z_{p+1},first
// (primes: next chunk). Three launches: local interior solves (parallel over chunks and wavenumbers),
// the separator system (parallel over wavenumbers), the correction. The result equals the sequential
// Thomas solve up to round-off; T, g, h depend only on (chunk type, wavenumber) and are tabulated.
// Tables (type 0 = first chunk, whose first row carries the x- Neumann change; type 1 = the others),
// each [type][r][j], r < kChunk-1: c (Thomas factors), g, h.
// ---------------------------------------------------------------------------------------------
constexpr int kChunk = 32;

// cback: the table again, read by the back substitution through a second pointer so that the compiler loads
// the factors again instead of keeping all 31 forward-sweep factors live in registers (198 registers and one
// CTA of 256 threads per SM that way; with the reload and a cap of 168 registers, three CTAs of 128 threads).
template <typename T>
__global__ void __launch_bounds__(128, 3) k_chase_local(T* __restrict__ f, int nx, int ny, long long batch,
                                                        const T* __restrict__ ctab, const T* __restrict__ cback,
                                                        T* __restrict__ zend, int skip_last)
{
    constexpr int  Li = kChunk - 1;
    const int      P  = nx / kChunk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= batch * P * ny) return;
    const int       j   = (int)(t % ny);
    if (skip_last && j == ny - 1) return;
    const long long bp  = t / ny;
    const int       p   = (int)(bp % P);
    const long long b   = bp / P;
    const int       typ = p == 0 ? 0 : 1;
    T*              col = f + b * (long long)nx * ny + (long long)p * kChunk * ny + j;
    const T*        c   = ctab + (long long)typ * Li * ny + j;
    const T*        cb  = cback + (long long)typ * Li * ny + j;
    T               y[Li];
#pragma unroll
    for (int r = 0; r < Li; ++r) y[r] = col[(long long)r * ny];
    T prev = 0;
#pragma unroll
    for (int r = 0; r < Li; ++r)
    {
        prev = (y[r] - prev) * __ldg(c + (long long)r * ny);
        y[r] = prev;
    }
#pragma unroll
    for (int r = Li - 2; r >= 0; --r) y[r] = y[r] - __ldg(cb + (long long)r * ny) * y[r + 1];
#pragma unroll
    for (int r = 0; r < Li; ++r) col[(long long)r * ny] = y[r];
    T* ze                      = zend + ((b * P + p) * 2) * (long long)ny + j;
    ze[0]                      = y[0];
    ze[ny]                     = y[Li - 1];
}

// Separator system per (field, wavenumber). ends: [type][4][j] = g_first, g_last, h_first, h_last.
// Its matrix depends on the wavenumber only, so the Thomas factors of every row but the last are tabulated
// (scp: c_p, sid: 1 / den_p; see separator_factors); the last row (which depends on P and the x+ Neumann
// end) is formed here from c_{P-2}. Per solve the forward elimination y_p = (rhs_p - lower y_{p-1}) sid_p
// and the back substitution x_p = y_p - c_p x_{p+1} are affine recurrences along p, evaluated as a blocked
// scan: a CTA takes 32 wavenumbers of one field (lane = j, every access coalesced along j) and splits the
// separators into kRedWarps contiguous ranges, one per warp; each warp composes the maps of its range, the
// CTA combines the compositions of the ranges before (after) it through shared memory, and the warp walks
// its range from that incoming value. work: P values per (field, wavenumber), the forward map slopes.
constexpr int kRedWarps = 8;

template <typename T>
__global__ void __launch_bounds__(32 * kRedWarps) k_chase_reduced(T* __restrict__ f, int nx, int ny, long long batch,
                                                                  const T* __restrict__ ends, const T* __restrict__ dsep,
                                                                  int end_neumann, const T* __restrict__ zend,
                                                                  T* __restrict__ bsep, T* __restrict__ work,
                                                                  const T* __restrict__ scp, const T* __restrict__ sid,
                                                                  int skip_last)
{
    constexpr int   kAhead = 8;
    __shared__ T    sa[kRedWarps][32], sb[kRedWarps][32];
    const int       tiles = (ny + 31) / 32;
    const long long b     = blockIdx.x / tiles;
    if (b >= batch) return;  // uniform over the CTA
    const int  lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int  j0   = (int)(blockIdx.x % tiles) * 32 + lane;
    const bool act  = j0 < ny && !(skip_last && j0 == ny - 1);
    const int  j    = j0 < ny ? j0 : 0;  // idle lanes compute on column 0 and store nothing
    const int  P    = nx / kChunk;
    const int  per  = (P + kRedWarps - 1) / kRedWarps;
    const int  pb = min(P, w * per), pe = min(P, pb + per);
    const T    e1_1 = ends[(1 * 4 + 1) * (long long)ny + j];
    const T*   ze   = zend + b * (long long)P * 2 * ny + j;
    T*         bs   = bsep + b * (long long)P * ny + j;  // B_p, then y_p, then the solution x_p
    T*         wk   = work + b * (long long)P * ny + j;  // A_p of y_p = A_p y_{p-1} + B_p
    T*         fb   = f + b * (long long)nx * ny + j;

    T ca = 1, cb = 0;
    for (int p0 = pb; p0 < pe; p0 += kAhead)
    {
        T rhs_v[kAhead], inv_v[kAhead];
#pragma unroll
        for (int q = 0; q < kAhead; ++q)
        {
            const int p = p0 + q;
            if (p >= pe) break;
            T r = fb[(long long)(p * kChunk + kChunk - 1) * ny] - ze[(long long)(2 * p + 1) * ny];
            if (p < P - 1) r -= ze[(long long)(2 * (p + 1)) * ny];
            rhs_v[q] = r;
            if (p < P - 1) inv_v[q] = sid[(long long)p * ny + j];
            else  // last row: no next chunk, x+ Neumann end
            {
                const T lower = p > 0 ? -e1_1 : (T)0;
                const T diag  = (end_neumann ? dsep[j] + (T)1 : dsep[j]) -
                               (p == 0 ? ends[(0 * 4 + 3) * (long long)ny + j] : ends[(1 * 4 + 3) * (long long)ny + j]);
                inv_v[q] = (T)1 / (diag - lower * (p > 0 ? scp[(long long)(p - 1) * ny + j] : (T)0));
            }
        }
#pragma unroll
        for (int q = 0; q < kAhead; ++q)
        {
            const int p = p0 + q;
            if (p >= pe) break;
            const T A = p > 0 ? e1_1 * inv_v[q] : (T)0;  // -lower inv
            const T B = rhs_v[q] * inv_v[q];
            if (act)
            {
                wk[(long long)p * ny] = A;
                bs[(long long)p * ny] = B;
            }
            cb = A * cb + B;
            ca = A * ca;
        }
    }
    sa[w][lane] = ca;
    sb[w][lane] = cb;
    __syncthreads();
    T y = 0;  // y_{pb-1}
    for (int v = 0; v < w; ++v) y = sa[v][lane] * y + sb[v][lane];
    for (int p = pb; p < pe; ++p)
    {
        const T A = act ? wk[(long long)p * ny] : (T)0, B = act ? bs[(long long)p * ny] : (T)0;
        y         = A * y + B;
        if (act) bs[(long long)p * ny] = y;
    }
    __syncthreads();  // every warp has read the forward compositions

    ca = 1;
    cb = 0;
    for (int p = pe - 1; p >= pb; --p)  // x_p = -c_p x_{p+1} + y_p, c_{P-1} = 0
    {
        const T c  = p < P - 1 ? scp[(long long)p * ny + j] : (T)0;
        const T yp = act ? bs[(long long)p * ny] : (T)0;
        cb         = -c * cb + yp;
        ca         = -c * ca;
    }
    sa[w][lane] = ca;
    sb[w][lane] = cb;
    __syncthreads();
    T x = 0;  // x_{pe}
    for (int v = kRedWarps - 1; v > w; --v) x = sa[v][lane] * x + sb[v][lane];
    for (int p = pe - 1; p >= pb; --p)
    {
        const T c  = p < P - 1 ? scp[(long long)p * ny + j] : (T)0;
        const T yp = act ? bs[(long long)p * ny] : (T)0;
        x          = yp - c * x;
        if (act)
        {
            bs[(long long)p * ny]                          = x;  // the correction pass reads it
            fb[(long long)(p * kChunk + kChunk - 1) * ny] = x;
        }
    }
}

// x_int = z - B_{p-1} g - B_p h on the interior rows.
template <typename T>
__global__ void __launch_bounds__(256) k_chase_correct(T* __restrict__ f, int nx, int ny, long long batch,
                                                       const T* __restrict__ gtab, const T* __restrict__ htab,
                                                       const T* __restrict__ bsep, int skip_last)
{
    constexpr int  Li = kChunk - 1;
    const int      P  = nx / kChunk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= batch * P * ny) return;
    const int       j   = (int)(t % ny);
    if (skip_last && j == ny - 1) return;
    const long long bp  = t / ny;
    const int       p   = (int)(bp % P);
    const long long b   = bp / P;
    const int       typ = p == 0 ? 0 : 1;
    const T*        bs  = bsep + b * (long long)P * ny + j;
    const T         bl  = p > 0 ? bs[(long long)(p - 1) * ny] : (T)0;
    const T         br  = bs[(long long)p * ny];
    T*              col = f + b * (long long)nx * ny + (long long)p * kChunk * ny + j;
    const T*        g   = gtab + (long long)typ * Li * ny + j;
    const T*        h   = htab + (long long)typ * Li * ny + j;
#pragma unroll 8
    for (int r = 0; r < Li; ++r)
    {
        const long long o = (long long)r * ny;
        col[o]            = col[o] - bl * __ldg(g + o) - br * __ldg(h + o);
    }
}

}  // namespace fpb
