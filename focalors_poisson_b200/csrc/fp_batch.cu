// Batched composite solves (fp_batch.h). Host plan + heterogeneous persistent kernels.
#include "fp_batch.h"
#include "fp_chase.cuh"
#include "fp_ops.cuh"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <type_traits>

namespace fpb
{

// =============================================================================================
// Device side
// =============================================================================================

// sqrt(2/(n+1)) sin(pi (k+1)(j+1)/(n+1)): DST-I basis vector k at point j (the reference's DD transform,
// pe/poisson/poisson_fft2d.cpp:19-57, is this orthonormal matrix).
__device__ __forceinline__ double dst_basis(int n, int k, int j)
{
    const long long q = (long long)(k + 1) * (j + 1) % (2LL * (n + 1));
    return sqrt(2.0 / (n + 1)) * sinpi((double)q / (double)(n + 1));
}

// ---------------------------------------------------------------------------------------------
// Partition chase (fp_chase.cuh) over many subdomains, out of place, with right-hand-side
// modifiers: rhs(i, k) = in(i, k) + sum_rows [i == row] c v[k] + sum_cols c s[i] psi_k(j)
// (a row term is a spectral vector on one row; a column term is a physical column of values at
// column j, whose y-DST is s[i] psi_k(j)).
// Rows are stored in T (FP64, or FP32 in the reduced-precision inner solves); the elimination itself,
// its tables and its scratch are FP64 for both. The lowest wavenumbers' tridiagonal systems are nearly
// singular (diagonal -2 - O(h^2), condition ~ nx^2): eliminated in FP32 they lose about 2 of FP32's 7
// digits (rel. error ~1e-2 at nx = 2048), in FP64 the FP32-rounded input is solved to ~1e-12, so an
// FP32-storage inner solve keeps FP32 accuracy (~1e-7) and refinement needs fewer steps.
// ---------------------------------------------------------------------------------------------
constexpr int kMaxMods = 4;

struct ChaseTabDev
{
    const double* cc;
    const double* cg;
    const double* chh;
    const double* cends;
    const double* dsep;
    int           end_neu;  // x+ face Neumann: last separator diagonal d + 1 (x- Neumann is in the type-0 tables)
    const double* scp;      // separator Thomas factors c_p [p][j] (rows not last)
    const double* sid;      // 1 / den_p [p][j]
    const double* cc_back;  // a copy of cc read by the back substitution (see k_b_chase_local)
};

template <typename T> struct ChaseSeg
{
    const T* in;
    T*       out;
    int      nx, ny, tab;
    double*  zend;  // scratch: 2 P ny
    double*  bsep;  // P ny
    double*  work;  // P ny
    int      nrow, ncol;
    int      row_i[kMaxMods];
    const double* row_v[kMaxMods];
    double   row_c[kMaxMods];
    int      col_j[kMaxMods];
    const double* col_s[kMaxMods];
    const double* col_tab[kMaxMods];  // y-basis values at column col_j (null: the DST-I basis)
    double   col_c[kMaxMods];
};

template <typename T> struct ModCtx
{
    double psi[kMaxMods];
};

template <typename T>
__device__ __forceinline__ void mod_init(const ChaseSeg<T>* __restrict__ sg, int ncol, int k, ModCtx<T>& m)
{
    for (int c = 0; c < ncol; ++c)
        m.psi[c] = sg->col_c[c] * (sg->col_tab[c] ? sg->col_tab[c][k] : dst_basis(sg->ny, k, sg->col_j[c]));
}
template <typename T>
__device__ __forceinline__ double mod_rhs(const ChaseSeg<T>* __restrict__ sg, int nrow, int ncol, const ModCtx<T>& m,
                                          int i, int k, double v)
{
    for (int r = 0; r < nrow; ++r)
        if (sg->row_i[r] == i) v += sg->row_c[r] * sg->row_v[r][k];
    for (int c = 0; c < ncol; ++c) v += m.psi[c] * sg->col_s[c][i];
    return v;
}

// blocks of segment s: prefix (in blocks); per segment P*ny threads (local / correct) or ny (reduced)
// Interior rows of the chunks. Modifiers: a row term can only fall on interior row 0 of chunk 0 (row
// nx-1 is the last separator, handled by k_b_chase_reduced); column terms add s_c[i] psi_c(j) to every
// row, applied as one pass per term over the thread's 31 rows.
// The back substitution reads its factors from a second copy of the table: from the same addresses the
// compiler keeps all 31 forward-sweep factors live in registers until the backward sweep (158 registers,
// 3 CTAs of 128 threads per SM); from a distinct array it loads them again, and two CTAs of 256 threads fit.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_b_chase_local(const ChaseSeg<T>* __restrict__ segs,
                                                       const long long* __restrict__ prefix, int nseg,
                                                       const ChaseTabDev* __restrict__ tabs)
{
    constexpr int      Li = kChunk - 1;
    const int          s  = seg_of(prefix, nseg, blockIdx.x);
    const ChaseSeg<T>* sg = segs + s;
    const int          ny = sg->ny, P = sg->nx / kChunk;
    const int          t  = (int)(blockIdx.x - prefix[s]) * blockDim.x + threadIdx.x;
    if (t >= P * ny) return;
    const int     j   = t % ny, p = t / ny;
    const int     typ = p == 0 ? 0 : 1;
    const T*      col = sg->in + (long long)p * kChunk * ny + j;
    T*            out = sg->out + (long long)p * kChunk * ny + j;
    const double* c   = tabs[sg->tab].cc + (long long)typ * Li * ny + j;
    const double* cb  = tabs[sg->tab].cc_back + (long long)typ * Li * ny + j;
    double        y[Li];
#pragma unroll
    for (int r = 0; r < Li; ++r) y[r] = (double)col[(long long)r * ny];
    const int ncol = sg->ncol;
    for (int q = 0; q < ncol; ++q)
    {
        const double  ps = sg->col_c[q] * (sg->col_tab[q] ? sg->col_tab[q][j] : dst_basis(ny, j, sg->col_j[q]));
        const double* sv = sg->col_s[q] + p * kChunk;
#pragma unroll
        for (int r = 0; r < Li; ++r) y[r] += ps * sv[r];
    }
    if (p == 0)
        for (int q = 0; q < sg->nrow; ++q)
            if (sg->row_i[q] == 0) y[0] += sg->row_c[q] * sg->row_v[q][j];
    double prev = 0;
#pragma unroll
    for (int r = 0; r < Li; ++r)
    {
        prev = (y[r] - prev) * __ldg(c + (long long)r * ny);
        y[r] = prev;
    }
#pragma unroll
    for (int r = Li - 2; r >= 0; --r) y[r] = y[r] - __ldg(cb + (long long)r * ny) * y[r + 1];
#pragma unroll
    for (int r = 0; r < Li; ++r) out[(long long)r * ny] = (T)y[r];
    double* ze = sg->zend + (long long)(p * 2) * ny + j;
    ze[0]      = y[0];
    ze[ny]     = y[Li - 1];
}

// Separator system per subdomain and wavenumber (the system of k_chase_reduced, tabulated Thomas factors
// for every row but the last). Per wavenumber j the forward elimination y_p = (rhs_p - lower y_{p-1}) inv_p
// and the back substitution x_p = y_p - scp_p x_{p+1} (p = 0..P-1, one separator per chunk) are affine
// recurrences along p. A CTA takes 32 wavenumbers (lane = j, so every access is coalesced along j) and
// splits the separators into kRedWarps contiguous ranges, one per warp: each warp composes the maps of its
// range, the CTA combines the compositions of the ranges before (after) it through shared memory, and the
// warp walks its range from that incoming value. The dependent chain per thread is P / kRedWarps maps per
// sweep instead of P memory round trips; the maps are the sequential ones, composed in another order.

template <typename T>
__global__ void __launch_bounds__(32 * kRedWarps) k_b_chase_reduced(const ChaseSeg<T>* __restrict__ segs,
                                                                    const long long* __restrict__ prefix, int nseg,
                                                                    const ChaseTabDev* __restrict__ tabs)
{
    constexpr int      kAhead = 8;
    __shared__ double  sa[kRedWarps][32], sb[kRedWarps][32];
    const int          s    = seg_of(prefix, nseg, blockIdx.x);
    const ChaseSeg<T>* sg   = segs + s;
    const int          ny   = sg->ny, nx = sg->nx, P = nx / kChunk;
    const int          lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int          j0   = (int)(blockIdx.x - prefix[s]) * 32 + lane;
    const bool         act  = j0 < ny;
    const int          j    = act ? j0 : 0;  // idle lanes compute on column 0 and store nothing
    const int          per  = (P + kRedWarps - 1) / kRedWarps;
    const int          pb = min(P, w * per), pe = min(P, pb + per);
    const ChaseTabDev tb   = tabs[sg->tab];
    const int            nrow = sg->nrow, ncol = sg->ncol;
    ModCtx<T>            mc;
    if (ncol > 0)  // column-term weights of the CTA's 32 wavenumbers: computed once (warp 0), shared
    {
        __shared__ double spsi[kMaxMods][32];
        if (w == 0)
        {
            mod_init(sg, ncol, j, mc);
            for (int c = 0; c < ncol; ++c) spsi[c][lane] = mc.psi[c];
        }
        __syncthreads();
        for (int c = 0; c < ncol; ++c) mc.psi[c] = spsi[c][lane];
    }
    const double  e1_1 = tb.cends[(1 * 4 + 1) * (long long)ny + j];
    const double* ze   = sg->zend + j;
    const T*      in   = sg->in;
    double*       bs   = sg->bsep + j;  // y_p, then x_p (the correction pass reads x)
    double*       wk   = sg->work + j;  // A_p of y_p = A_p y_{p-1} + B_p

    // forward maps of the range: A_p = -lower inv_p, B_p = rhs_p inv_p (B kept in bs), composed in (ca, cb)
    double ca = 1, cb = 0;
    for (int p0 = pb; p0 < pe; p0 += kAhead)
    {
        double rhs_v[kAhead], inv_v[kAhead];
#pragma unroll
        for (int q = 0; q < kAhead; ++q)
        {
            const int p = p0 + q;
            if (p >= pe) break;
            const int isep = p * kChunk + kChunk - 1;
            double r = mod_rhs(sg, nrow, ncol, mc, isep, j, (double)in[(long long)isep * ny + j]) -
                       ze[(long long)(2 * p + 1) * ny];
            if (p < P - 1) r -= ze[(long long)(2 * (p + 1)) * ny];
            rhs_v[q] = r;
            if (p < P - 1) inv_v[q] = tb.sid[(long long)p * ny + j];
            else  // last row: no next chunk, x+ Neumann end
            {
                const double lower = p > 0 ? -e1_1 : 0.0;
                const double diag  = (tb.end_neu ? tb.dsep[j] + 1.0 : tb.dsep[j]) -
                                    (p == 0 ? tb.cends[(0 * 4 + 3) * (long long)ny + j]
                                            : tb.cends[(1 * 4 + 3) * (long long)ny + j]);
                inv_v[q] = 1.0 / (diag - lower * (p > 0 ? tb.scp[(long long)(p - 1) * ny + j] : 0.0));
            }
        }
#pragma unroll
        for (int q = 0; q < kAhead; ++q)
        {
            const int p = p0 + q;
            if (p >= pe) break;
            const double A = p > 0 ? e1_1 * inv_v[q] : 0.0;  // -lower inv
            const double B = rhs_v[q] * inv_v[q];
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
    double y = 0;  // y_{pb-1}
    for (int v = 0; v < w; ++v) y = sa[v][lane] * y + sb[v][lane];
    for (int p = pb; p < pe; ++p)
    {
        const double A = act ? wk[(long long)p * ny] : 0.0, B = act ? bs[(long long)p * ny] : 0.0;
        y         = A * y + B;
        if (act) bs[(long long)p * ny] = y;
    }
    __syncthreads();  // every warp has read the forward compositions

    // back substitution maps x_p = -c_p x_{p+1} + y_p (c_{P-1} = 0), composed from the top of the range down
    ca = 1;
    cb = 0;
    for (int p = pe - 1; p >= pb; --p)
    {
        const double c  = p < P - 1 ? tb.scp[(long long)p * ny + j] : 0.0;
        const double yp = act ? bs[(long long)p * ny] : 0.0;
        cb              = -c * cb + yp;
        ca         = -c * ca;
    }
    sa[w][lane] = ca;
    sb[w][lane] = cb;
    __syncthreads();
    double x = 0;  // x_{pe}
    for (int v = kRedWarps - 1; v > w; --v) x = sa[v][lane] * x + sb[v][lane];
    for (int p = pe - 1; p >= pb; --p)
    {
        const double c  = p < P - 1 ? tb.scp[(long long)p * ny + j] : 0.0;
        const double yp = act ? bs[(long long)p * ny] : 0.0;
        x               = yp - c * x;
        if (act)
        {
            bs[(long long)p * ny] = x;
            sg->out[(long long)(p * kChunk + kChunk - 1) * ny + j] = (T)x;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_b_chase_correct(const ChaseSeg<T>* __restrict__ segs,
                                                         const long long* __restrict__ prefix, int nseg,
                                                         const ChaseTabDev* __restrict__ tabs)
{
    constexpr int      Li = kChunk - 1;
    const int          s  = seg_of(prefix, nseg, blockIdx.x);
    const ChaseSeg<T>* sg = segs + s;
    const int          ny = sg->ny, P = sg->nx / kChunk;
    const int          t  = (int)(blockIdx.x - prefix[s]) * blockDim.x + threadIdx.x;
    if (t >= P * ny) return;
    const int            j   = t % ny, p = t / ny;
    const int            typ = p == 0 ? 0 : 1;
    const ChaseTabDev tb  = tabs[sg->tab];
    const double*     bs  = sg->bsep + j;
    const double      bl  = p > 0 ? bs[(long long)(p - 1) * ny] : 0.0;
    const double      br  = bs[(long long)p * ny];
    T*                col = sg->out + (long long)p * kChunk * ny + j;
    const double*     g   = tb.cg + (long long)typ * Li * ny + j;
    const double*     h   = tb.chh + (long long)typ * Li * ny + j;
#pragma unroll 8
    for (int r = 0; r < Li; ++r)
    {
        const long long o = (long long)r * ny;
        col[o]            = (T)((double)col[o] - bl * __ldg(g + o) - br * __ldg(h + o));
    }
}

// ---------------------------------------------------------------------------------------------
// Small per-subdomain / per-problem kernels
// ---------------------------------------------------------------------------------------------
// out[i] = coef * sum_k psi_k(j) X(i, k): the physical value at column j of a y-spectral field.
template <typename T> struct ColReq
{
    const T*      X;
    int           nx, ny, j;
    double*       out;
    double        coef;
    const double* tab;  // y-basis values at column j (null: the DST-I basis)
};
template <typename T>
__global__ void k_b_colvals(const ColReq<T>* __restrict__ reqs, const long long* __restrict__ prefix, int nreq)
{
    const long long w    = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int       lane = threadIdx.x & 31;
    if (w >= prefix[nreq]) return;
    const int       q = seg_of(prefix, nreq, w);
    const ColReq<T> R = reqs[q];
    const int       i = (int)(w - prefix[q]);
    const T*        row = R.X + (long long)i * R.ny;
    double          acc = 0;
    constexpr int   U   = 8;  // elements per lane loaded ahead of the (in-order) accumulation
    for (int k0 = lane; k0 < R.ny; k0 += 32 * U)
    {
        double xv[U], bv[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int k = k0 + 32 * u;
            xv[u]       = k < R.ny ? (double)row[k] : 0.0;
            bv[u]       = k < R.ny ? (R.tab ? R.tab[k] : dst_basis(R.ny, k, R.j)) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) acc += bv[u] * xv[u];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) R.out[i] = R.coef * acc;
}

// out[k] = coef * X(i, k)
template <typename T> struct RowReq
{
    const T* X;
    int      ny, i;
    double*  out;
    double   coef;
};
template <typename T>
__global__ void k_b_rowcopy(const RowReq<T>* __restrict__ reqs, const long long* __restrict__ prefix, int nreq)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= prefix[nreq]) return;
    const int       q = seg_of(prefix, nreq, t);
    const RowReq<T> R = reqs[q];
    const int       k = (int)(t - prefix[q]);
    R.out[k]          = R.coef * (double)R.X[(long long)R.i * R.ny + k];
}

// Interface solve of one problem in the spectral bases (see fp_batch.h). Edges: x-edges e (root faces
// x- / x+, rows ie[e]) with y-spectral unknowns (ny), y-edges Y (root faces y- / y+, columns jy[Y]) with
// x-spectral unknowns (nx).
struct BIface
{
    int           nx, ny, nxe, nye;
    int           ie[2], jy[2];
    double        r;
    const double* alpha;  // nx: x eigenvalues - 2 ... (root)
    const double* beta;   // ny
    const double* sig[2];   // x-edge leaf responses (ny)
    const double* sigp[2];  // y-edge leaf responses (nx)
    const double* invxx;    // ny blocks of nxe x nxe
    const double* invyy;    // nx blocks of nye x nye (used when nxe == 0)
    const double* rinv;     // (nye nx)^2 column-major (when nxe > 0 and nye > 0)
    double*       gX;   // nxe * ny
    double*       gY;   // nye * nx (x-spectral)
    double*       zX;   // nxe * ny
    double*       rhsY; // nye * nx
    double*       yX;   // nxe * ny
    double*       yY;   // nye * nx (x-spectral)
    double*       sY;   // nye * nx: sigma' yY (x-spectral)
    double*       bX;   // nxe * ny: -leaf edge rows (y-spectral), root right-hand side terms
    double*       bX2;  // nxe * ny: bX + sigma yX
    const double* K;    // nx * ny: K[m ny + k] = 1 / (alpha_m + r beta_k), the root's inverse in the 2D basis
    double*       vxy;  // [e][Y] ny: psi_k(jY) sig_e[k] zX[e][k]
    double*       wxy;  // [e][Y] nx: chi_m(ie) sig'_Y[m] yY[Y][m]
    int           yy_chunks, yx_chunks;  // column chunks of the two dense products (both edge kinds)
    double*       part_yy;  // [chunk][nye nx] partial sums of Rinv rhsY
    double*       part_yx;  // [chunk][e*2+Y][ny] partial sums of K^T wxy
};

// Dense products of the interface solve run as 32-row tiles x column chunks, 8 warps per tile splitting
// the chunk's columns; partial sums are added in a fixed order by the finishing kernel (reproducible).
constexpr int kIfTile = 32, kIfWarps = 8, kIfChunkYY = 1024, kIfChunkYX = 128;

__device__ __forceinline__ double chi_edge(int n, int m, int i) { return dst_basis(n, m, i); }

// zX = invXX gX, thread per (problem, k)
__global__ void k_if_zx(const BIface* __restrict__ P, const long long* __restrict__ prefix, int np)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= prefix[np]) return;
    const int    p = seg_of(prefix, np, t);
    const BIface F = P[p];
    const int    k = (int)(t - prefix[p]);
    const int    E = F.nxe;
    const double* B = F.invxx + (long long)k * E * E;
    for (int e = 0; e < E; ++e)
    {
        double v = 0;
        for (int e2 = 0; e2 < E; ++e2) v += B[e * E + e2] * F.gX[e2 * F.ny + k];
        F.zX[e * F.ny + k] = v;
        for (int Y = 0; Y < F.nye; ++Y)
            F.vxy[(e * 2 + Y) * F.ny + k] = dst_basis(F.ny, k, F.jy[Y]) * F.sig[e][k] * v;
    }
}

// rhsY[Y][m] = gY[Y][m] + sum_{e,k} chi_m(ie) psi_k(jY) sig_e[k] zX[e][k] / (alpha_m + r beta_k);
// warp per (problem, Y, m)
__global__ void k_if_rhsy(const BIface* __restrict__ P, const long long* __restrict__ prefix, int np)
{
    const long long w    = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int       lane = threadIdx.x & 31;
    if (w >= prefix[np]) return;
    const int     p  = seg_of(prefix, np, w);
    const BIface& F  = P[p];
    const int     q  = (int)(w - prefix[p]);
    const int     Y  = q / F.nx, m = q - Y * F.nx;
    double        acc = 0;
    for (int e = 0; e < F.nxe; ++e)
    {
        const double* Km = F.K + (long long)m * F.ny;
        const double* v  = F.vxy + (e * 2 + Y) * F.ny;
        double        a  = 0;
        for (int k = lane; k < F.ny; k += 32) a += Km[k] * v[k];
        acc += chi_edge(F.nx, m, F.ie[e]) * a;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) F.rhsY[Y * F.nx + m] = F.gY[Y * F.nx + m] + acc;
}

// Partial sums of yY = Rinv rhsY (problems with both edge kinds): block = (row tile, column chunk); lane =
// row (Rinv is column-major: a warp reads 32 consecutive rows of one column), warp = every 8th column.
__global__ void __launch_bounds__(256) k_if_yy_part(const BIface* __restrict__ P, const long long* __restrict__ prefix,
                                                    int np)
{
    __shared__ double red[kIfWarps][kIfTile];
    const int     p    = seg_of(prefix, np, blockIdx.x);
    const BIface& F    = P[p];
    const int     b    = (int)(blockIdx.x - prefix[p]);
    const int     tile = b / F.yy_chunks, chunk = b - tile * F.yy_chunks;
    const int     lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int     n    = F.nye * F.nx;
    const int     q    = tile * kIfTile + lane;
    const int     c1   = min(n, (chunk + 1) * kIfChunkYY);
    const double* rinv = F.rinv;
    const double* rhs  = F.rhsY;
    double        acc  = 0;
    if (q < n)
#pragma unroll 4
        for (int c = chunk * kIfChunkYY + warp; c < c1; c += kIfWarps) acc += rinv[(long long)c * n + q] * rhs[c];
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && q < n)
    {
        double v = 0;
        for (int w = 0; w < kIfWarps; ++w) v += red[w][lane];
        F.part_yy[(long long)chunk * n + q] = v;
    }
}

// yY (sum of the partials, or the per-m blocks without x-edges); sY = sigma' yY; wxy for the yx product
__global__ void k_if_yy(const BIface* __restrict__ P, const long long* __restrict__ prefix, int np)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= prefix[np]) return;
    const int     p = seg_of(prefix, np, t);
    const BIface& F = P[p];
    const int     q = (int)(t - prefix[p]);  // row of the nye*nx system
    const int     n = F.nye * F.nx;
    double        v = 0;
    if (F.nxe > 0)
    {
        for (int c = 0; c < F.yy_chunks; ++c) v += F.part_yy[(long long)c * n + q];
    }
    else
    {
        const int Y = q / F.nx, m = q - Y * F.nx, E = F.nye;
        const double* B = F.invyy + (long long)m * E * E;
        for (int Y2 = 0; Y2 < E; ++Y2) v += B[Y * E + Y2] * F.rhsY[Y2 * F.nx + m];
    }
    F.yY[q] = v;
    const int Y = q / F.nx, m = q - Y * F.nx;
    F.sY[q]    = F.sigp[Y][m] * v;
    for (int e = 0; e < F.nxe; ++e) F.wxy[(e * 2 + Y) * F.nx + m] = chi_edge(F.nx, m, F.ie[e]) * F.sY[q];
}

// Partial sums of sum_m K[m][k] wxy[e][Y][m] (problems with both edge kinds): block = (k tile, m chunk);
// lane = k (a warp reads 32 consecutive k of one K row), warp = every 8th m.
__global__ void __launch_bounds__(256) k_if_yx_part(const BIface* __restrict__ P, const long long* __restrict__ prefix,
                                                    int np)
{
    __shared__ double red[kIfWarps][4][kIfTile];
    const int     p    = seg_of(prefix, np, blockIdx.x);
    const BIface& F    = P[p];
    const int     b    = (int)(blockIdx.x - prefix[p]);
    const int     tile = b / F.yx_chunks, chunk = b - tile * F.yx_chunks;
    const int     lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int     k    = tile * kIfTile + lane;
    const int     nx = F.nx, ny = F.ny, nxe = F.nxe, nye = F.nye;
    const int     m1   = min(nx, (chunk + 1) * kIfChunkYX);
    const double* Kp   = F.K;
    const double* wxy  = F.wxy;
    double        acc[4] = {0, 0, 0, 0};  // [e*2+Y], static indices so they stay in registers
    if (k < ny)
#pragma unroll 4
        for (int m = chunk * kIfChunkYX + warp; m < m1; m += kIfWarps)
        {
            const double Kmk = Kp[(long long)m * ny + k];
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
                for (int Y = 0; Y < 2; ++Y)
                    if (e < nxe && Y < nye) acc[e * 2 + Y] += Kmk * wxy[(e * 2 + Y) * nx + m];
        }
    for (int i = 0; i < 4; ++i) red[warp][i][lane] = acc[i];
    __syncthreads();
    if (warp == 0 && k < F.ny)
        for (int i = 0; i < 4; ++i)
        {
            double v = 0;
            for (int w = 0; w < kIfWarps; ++w) v += red[w][i][lane];
            F.part_yx[((long long)chunk * 4 + i) * F.ny + k] = v;
        }
}

// yX[e][k] = sum_e' invXX_k(e, e') (gX[e'][k] + sum_Y psi_k(jY) sum_m K[m][k] wxy[e'][Y][m]); bX2 = bX + sig yX.
__global__ void k_if_yx(const BIface* __restrict__ P, const long long* __restrict__ prefix, int np)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= prefix[np]) return;
    const int     p = seg_of(prefix, np, t);
    const BIface& F = P[p];
    const int     k = (int)(t - prefix[p]);
    double        tt[2] = {0, 0};
    for (int Y = 0; Y < F.nye; ++Y)
    {
        const double pk = dst_basis(F.ny, k, F.jy[Y]);
        for (int e = 0; e < F.nxe; ++e)
        {
            double a = 0;
            for (int c = 0; c < F.yx_chunks; ++c) a += F.part_yx[((long long)c * 4 + e * 2 + Y) * F.ny + k];
            tt[e] += pk * a;
        }
    }
    const int     E = F.nxe;
    const double* B = F.invxx + (long long)k * E * E;
    for (int e = 0; e < E; ++e)
    {
        double v = 0;
        for (int e2 = 0; e2 < E; ++e2) v += B[e * E + e2] * (F.gX[e2 * F.ny + k] + tt[e2]);
        F.yX[e * F.ny + k]  = v;
        F.bX2[e * F.ny + k] = F.bX[e * F.ny + k] + F.sig[e][k] * v;
    }
}

// K[m ny + k] = 1 / (alpha_m + r beta_k) of one problem's root
__global__ void k_root_inverse(const BIface F, double* K)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)F.nx * F.ny) return;
    const int m = (int)(t / F.ny), k = (int)(t - (long long)m * F.ny);
    K[t]        = 1.0 / (F.alpha[m] + F.r * F.beta[k]);
}

// ---------------------------------------------------------------------------------------------
// Setup kernels: closed-form spectral responses
// ---------------------------------------------------------------------------------------------
// out[q] = sum_{m < n} w(m) / (eig_a[m] + rr * eig_b[q]), w(m) = chi_m(ia) chi_m(ib) over n points:
// the Green's function of a Dirichlet tridiagonal line between points ia and ib, per transverse mode q.
struct GreenReq
{
    int           n, ia, ib, nq;
    const double* eig_a;  // n
    const double* eig_b;  // nq
    double        rr;
    double*       out;    // nq
    const double* wts;    // n weights w(m) (null: the DST-I products chi_m(ia) chi_m(ib))
};
__global__ void k_green(const GreenReq* __restrict__ reqs, const long long* __restrict__ prefix, int nreq)
{
    const long long w    = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int       lane = threadIdx.x & 31;
    if (w >= prefix[nreq]) return;
    const int      q0 = seg_of(prefix, nreq, w);
    const GreenReq R  = reqs[q0];
    const int      q  = (int)(w - prefix[q0]);
    const double   b  = R.rr * R.eig_b[q];
    double         acc = 0;
    for (int m = lane; m < R.n; m += 32)
        acc += (R.wts ? R.wts[m] : dst_basis(R.n, m, R.ia) * dst_basis(R.n, m, R.ib)) / (R.eig_a[m] + b);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) R.out[q] = acc;
}

// out[k] = (T_k^-1)(i', i') for T_k = tridiag(1, D, 1) of n rows, D = d[k] (+1 on a Neumann end row):
// the response of a subdomain at its interface row i' (0 or n-1) to an impulse there, per y-mode k, by
// eliminating from the far end (a continued fraction).
struct EndReq
{
    int           n, at_start, neu_lo, neu_hi, nq;
    const double* d;
    double*       out;
};
__global__ void k_green_end(const EndReq* __restrict__ reqs, const long long* __restrict__ prefix, int nreq)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= prefix[nreq]) return;
    const int    q = seg_of(prefix, nreq, t);
    const EndReq R = reqs[q];
    const int    k = (int)(t - prefix[q]);
    const double d = R.d[k];
    auto D = [&](int i) { return d + ((i == 0 && R.neu_lo) || (i == R.n - 1 && R.neu_hi) ? 1.0 : 0.0); };
    double c = 0.0;
    if (R.at_start)
        for (int i = R.n - 1; i >= 1; --i) c = 1.0 / (D(i) - c);
    else
        for (int i = 0; i <= R.n - 2; ++i) c = 1.0 / (D(i) - c);
    R.out[k] = 1.0 / (D(R.at_start ? 0 : R.n - 1) - c);
}

// A[(Y,m),(e,k)] (column-major, ld = nY) and B[(e,k),(Y,m)] = sum_e' invXX_k(e,e') M_XY(e',k; Y,m)
// (column-major, ld = nX) of one problem, for R = M_YY - A B.
__global__ void k_cross_AB(const BIface F, double* A, double* B)
{
    const int       nY = F.nye * F.nx, nX = F.nxe * F.ny;
    const long long t  = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nY * nX) return;
    const int row = (int)(t % nY), col = (int)(t / nY);  // A: row (Y, m), col (e, k)
    {
        const int Y = row / F.nx, m = row - Y * F.nx, e = col / F.ny, k = col - e * F.ny;
        A[(long long)col * nY + row] = -chi_edge(F.nx, m, F.ie[e]) * dst_basis(F.ny, k, F.jy[Y]) * F.sig[e][k] /
                                       (F.alpha[m] + F.r * F.beta[k]);
    }
    {
        // B: row (e, k) = t % nX, col (Y, m) = t / nX
        const int brow = (int)(t % nX), bcol = (int)(t / nX);
        const int e = brow / F.ny, k = brow - e * F.ny, Y = bcol / F.nx, m = bcol - Y * F.nx;
        const int E = F.nxe;
        double    v = 0;
        for (int e2 = 0; e2 < E; ++e2)
            v += F.invxx[(long long)k * E * E + e * E + e2] *
                 (-chi_edge(F.nx, m, F.ie[e2]) * dst_basis(F.ny, k, F.jy[Y]) * F.sigp[Y][m] /
                  (F.alpha[m] + F.r * F.beta[k]));
        B[(long long)bcol * nX + brow] = v;
    }
}

// R = M_YY (column-major nY x nY): identity minus the per-m y-edge couplings H_m(jY, jY') sig'_Y'[m]
__global__ void k_myy(const BIface F, const double* H /* 2x2 blocks per m: H[(Y*2+Y2)*nx + m] */, double* R)
{
    const int       nY = F.nye * F.nx;
    const long long t  = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nY * nY) return;
    const int row = (int)(t % nY), col = (int)(t / nY);
    const int Y = row / F.nx, m = row - Y * F.nx, Y2 = col / F.nx, m2 = col - Y2 * F.nx;
    double    v = (row == col) ? 1.0 : 0.0;
    if (m == m2) v -= H[(long long)(Y * 2 + Y2) * F.nx + m] * F.sigp[Y2][m];
    R[t] = v;
}

// ---------------------------------------------------------------------------------------------
// Elementwise over many subdomains
// ---------------------------------------------------------------------------------------------
constexpr int kAsmCells  = 1024;  // cells per block of k_b_assemble
constexpr int kElemCells = 1024;  // cells per block of the residual and add-with-norms kernels

struct AsmSeg
{
    double*      f;
    double*      copy;  // when non-null: copy = assembled f (f untouched)
    AssembleArgs a;
};
__global__ void k_b_assemble(const AsmSeg* __restrict__ segs, const long long* __restrict__ prefix, int nseg)
{
    const int     s    = seg_of(prefix, nseg, blockIdx.x);
    const AsmSeg* sg   = segs + s;
    const int     n    = sg->a.nx * sg->a.ny;
    const int     t0   = (int)(blockIdx.x - prefix[s]) * kAsmCells;
    const int     t1   = min(n, t0 + kAsmCells);
    double*       copy = sg->copy;
    double*       f    = sg->f;
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x)
    {
        if (copy)
        {
            copy[t] = f[t];
            assemble_at(copy, t, sg->a);
        }
        else
            assemble_at(f, t, sg->a);
    }
}

struct ResSeg
{
    double*       r;
    const double* fs;
    const double* u;
    ResidualArgs  a;
    double*       partial;  // per block: sum r^2 (or null)
    double*       partial_f;  // per block: sum fs^2 (or null)
};
__global__ void __launch_bounds__(256) k_b_residual(const ResSeg* __restrict__ segs, const long long* __restrict__ prefix,
                                                    int nseg)
{
    __shared__ double sh[32];
    const int     s  = seg_of(prefix, nseg, blockIdx.x);
    const ResSeg* sg = segs + s;
    const int     t0 = (int)(blockIdx.x - prefix[s]) * kElemCells;
    const int     t1 = min(sg->a.nx * sg->a.ny, t0 + kElemCells);
    double        rr = 0, ff = 0;
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x)
    {
        const double fs = sg->fs[t];
        const double v  = composite_residual_at(sg->u, fs, t, sg->a);
        if (sg->r) sg->r[t] = v;
        rr += v * v;
        ff += fs * fs;
    }
    if (sg->partial)
    {
        const double a = block_sum(rr, sh);
        __syncthreads();
        const double b = block_sum(ff, sh);
        if (threadIdx.x == 0)
        {
            sg->partial[blockIdx.x - prefix[s]]   = a;
            sg->partial_f[blockIdx.x - prefix[s]] = b;
        }
    }
}

// u (+)= c over many subdomains with per-block partial sums of c^2 and (new) u^2
struct AddSeg
{
    double*       u;
    const double* c;
    long long     n;
    double*       pc;  // per block
    double*       pu;
};
__global__ void __launch_bounds__(256) k_b_add_norms(const AddSeg* __restrict__ segs, const long long* __restrict__ prefix,
                                                     int nseg, int first)
{
    __shared__ double sh[32];
    const int     s  = seg_of(prefix, nseg, blockIdx.x);
    const AddSeg* sg = segs + s;
    const long long t0 = (blockIdx.x - prefix[s]) * (long long)kElemCells;
    const long long t1 = t0 + kElemCells < sg->n ? t0 + kElemCells : sg->n;
    double        cc = 0, uu = 0;
    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x)
    {
        const double c = sg->c[t];
        const double u = first ? c : sg->u[t] + c;
        sg->u[t]       = u;
        cc += c * c;
        uu += u * u;
    }
    const double a = block_sum(cc, sh);
    __syncthreads();
    const double b = block_sum(uu, sh);
    if (threadIdx.x == 0)
    {
        sg->pc[blockIdx.x - prefix[s]] = a;
        sg->pu[blockIdx.x - prefix[s]] = b;
    }
}

// State of a refinement run on the device (the refinement graph's loop control).
struct IrState
{
    int    steps;       // inner solves taken
    int    stop;        // the last check ended the loop
    int    err;         // non-finite correction or solution norm in this run
    int    err_sticky;  // the same over every run since the host last cleared it
    double change;      // last |correction| / |u|
    double last;        // the change before it
};

__global__ void k_ir_init(IrState* st)
{
    st->steps  = 1;  // the first inner solve wrote the solution itself
    st->stop   = 0;
    st->err    = 0;
    st->change = 1.0;
    st->last   = 0.0;
}

// After an add-with-norms pass: reduces its per-block partial sums (nb of |c|^2, then nb of |u|^2), applies the
// stop rule of the host loop (BatchImpl::refine) and sets the refinement graph's loop condition.
__global__ void __launch_bounds__(256) k_ir_check(const double* __restrict__ part, long long nb, IrState* st,
                                                  double rel_tol, int max_refine, cudaGraphConditionalHandle loop)
{
    __shared__ double sh[32];
    double            c = 0, u = 0;
    for (long long b = threadIdx.x; b < nb; b += blockDim.x)
    {
        c += part[b];
        u += part[nb + b];
    }
    const double cn = block_sum(c, sh);
    __syncthreads();
    const double un = block_sum(u, sh);
    if (threadIdx.x != 0) return;
    const int steps = st->steps + 1;
    st->steps       = steps;
    int stop        = steps >= max_refine;
    if (!isfinite(cn) || !isfinite(un))
    {
        st->err        = 1;
        st->err_sticky = 1;
        stop           = 1;
    }
    else
    {
        const double last   = st->change;
        const double change = un > 0 ? sqrt(cn / un) : 0.0;
        st->last            = last;
        st->change          = change;
        if (change <= rel_tol || (steps >= 2 && last > 0 && change * (change / last) <= rel_tol)) stop = 1;
    }
    st->stop = stop;
    cudaGraphSetConditional(loop, stop ? 0u : 1u);
}


// DST-I of a few rows of one length n as a dense product with the transform's matrix T (n x n, symmetric,
// T[k][i] = sqrt(2/(n+1)) sin(pi (k+1)(i+1) / (n+1)), the columns the FFT plan produces): one CTA of
// kEdgeMvThreads per output index k reads T's row k once for all the record's rows (four loads in flight per
// thread), then a block reduction. For the handful of interface vectors of a single problem this streams T
// once through the whole GPU where the FFT form runs one CTA per row, latency-bound.
constexpr int kEdgeMvRows    = 8;
constexpr int kEdgeMvThreads = 128;
struct EdgeMv
{
    const double* T;
    int           n, rows;
    const double* in[kEdgeMvRows];
    double*       out[kEdgeMvRows];
};
__global__ void __launch_bounds__(kEdgeMvThreads) k_edge_dst_mv(const EdgeMv* __restrict__ recs,
                                                                const long long* __restrict__ prefix, int nrec)
{
    __shared__ double sh[kEdgeMvRows][kEdgeMvThreads / 32];
    const int     s  = seg_of(prefix, nrec, blockIdx.x);
    const EdgeMv& r  = recs[s];
    const int     k  = (int)(blockIdx.x - prefix[s]);
    const double* Tk = r.T + (long long)k * r.n;
    double        acc[kEdgeMvRows];
#pragma unroll
    for (int q = 0; q < kEdgeMvRows; ++q) acc[q] = 0.0;
    for (int i0 = threadIdx.x; i0 < r.n; i0 += 4 * kEdgeMvThreads)
    {
        double t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            const int i = i0 + u * kEdgeMvThreads;
            t[u]        = i < r.n ? __ldg(Tk + i) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kEdgeMvRows; ++q)
            if (q < r.rows)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    const int i = i0 + u * kEdgeMvThreads;
                    if (i < r.n) acc[q] += t[u] * r.in[q][i];
                }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kEdgeMvRows; ++q)
    {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < r.rows)
    {
        double v = 0.0;
        for (int w = 0; w < kEdgeMvThreads / 32; ++w) v += sh[threadIdx.x][w];
        r.out[threadIdx.x][k] = v;
    }
}

}  // namespace fpb

// =============================================================================================
// Host side
// =============================================================================================
namespace fpb
{
namespace
{

struct Segments  // a device work list: records + block/item prefix
{
    DevBuf    recs, prefix;
    int       n     = 0;
    long long total = 0;  // items (or blocks, or threads) over all records
    template <typename R> void set(const std::vector<R>& r, const std::vector<long long>& counts)
    {
        n = (int)r.size();
        std::vector<long long> p(r.size() + 1, 0);
        for (size_t i = 0; i < r.size(); ++i) p[i + 1] = p[i] + counts[i];
        total  = p.back();
        recs   = upload(r);
        prefix = upload(p);
    }
    template <typename R> const R* as() const { return recs.as<R>(); }
    const long long*              pre() const { return prefix.as<long long>(); }
};

int grid_of(long long threads, int block) { return (int)std::max<long long>(1, (threads + block - 1) / block); }

int sm_count()
{
    static int v = [] {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n;
    }();
    return v;
}

template <typename T> struct PlanSet  // transform plans by (family, row length)
{
    std::map<std::pair<int, int>, int>            index;
    std::vector<std::unique_ptr<DevTransform<T>>> tr;
    DevBuf                                        dev;
    size_t                                        smem       = 0;
    bool                                          stage_only = false;  // plans on the stage engine only
    int get(int kind, int n)
    {
        auto key = std::make_pair(kind, n);
        auto it  = index.find(key);
        if (it != index.end()) return it->second;
        tr.emplace_back(new DevTransform<T>(kind, n, !stage_only));
        smem = std::max(smem, tr.back()->smem);
        return index[key] = (int)tr.size() - 1;
    }
    // Device arguments, two per plan: [2 p] forward, [2 p + 1] inverse.
    void finish()
    {
        std::vector<XformArgs<T>> v;
        for (auto& t : tr)
        {
            v.push_back(t->args(false));
            v.push_back(t->args(true));
        }
        dev = upload(v);
    }
};

// A transform work list split by family and engine: one launch per family for its stage-engine plans (the
// autotuned CTA shape, shared memory of the largest plan) and one per (family, length M) for its
// register-engine plans (M/16 threads per CTA).
struct XList
{
    struct Part
    {
        int      kind = 0;
        int      eng = 0, threads = 0;  // register engine: threads per CTA (stage engine: autotuned)
        size_t   smem = 0;
        int      plan = -1;  // the plan of every run, when they share one (launched with it by value)
        Segments seg;
    };
    std::vector<Part> parts;
    template <typename T> void set(const std::vector<DstSeg>& recs, const std::vector<int>& kinds, const PlanSet<T>& ps)
    {
        parts.clear();
        for (int k : {K_DD, K_ND, K_DN})
        {
            std::map<int, std::vector<size_t>> groups;  // -1: stage engine, else M of the register engine
            for (size_t i = 0; i < recs.size(); ++i)
                if (kinds[i] == k)
                {
                    const FftDesc& d = ps.tr[recs[i].plan]->fd;
                    groups[d.eng == 1 ? d.M : -1].push_back(i);
                }
            for (auto& g : groups)
            {
                std::vector<DstSeg>    r;
                std::vector<long long> c;
                size_t                 sm   = 0;
                int                    plan = recs[g.second[0]].plan;
                for (size_t i : g.second)
                {
                    r.push_back(recs[i]);
                    c.push_back((recs[i].rows + 1) / 2);
                    sm = std::max(sm, ps.tr[recs[i].plan]->smem);
                    if (recs[i].plan != plan) plan = -1;
                }
                parts.emplace_back();
                parts.back().kind    = k;
                parts.back().eng     = g.first > 0 ? 1 : 0;
                parts.back().threads = g.first > 0 ? g.first / 16 : 0;
                parts.back().smem    = sm;
                parts.back().plan    = plan;
                parts.back().seg.set(r, c);
            }
        }
    }
};

template <typename T, int K, int I, typename TIN, typename TOUT, bool ACC> void prep_x()
{
    allow_max_dynamic_smem((const void*)k_b_xform<T, K, I, TIN, TOUT, ACC, 0>);
    allow_max_dynamic_smem((const void*)k_b_xform<T, K, I, TIN, TOUT, ACC, 1>);
    allow_max_dynamic_smem((const void*)k_b_xform<T, K, I, TIN, TOUT, ACC, 0, true>);
    allow_max_dynamic_smem((const void*)k_xform_rc<T, K, I, TIN, TOUT, ACC, kXformStaticM>);
}

// Stage engine: the autotuned CTA shape (threads, CTAs per SM); register engine: `threads` per CTA and as
// many CTAs as are resident at once, each looping over items. plan >= 0: every run uses that plan, whose
// arguments then go to the kernel by value (the stage engine's k_b_xform, and k_xform_rc for register-engine
// plans of length kXformStaticM); otherwise the kernel reads each run's plan from the plan array.
template <typename T, int K, int I, typename TIN, typename TOUT, bool ACC>
void launch_x1(const Segments& sg, const PlanSet<T>& ps, const BatchTiming& tm, cudaStream_t s, size_t smem = 0,
               int eng = 0, int threads = 0, int plan = -1)
{
    if (sg.total == 0) return;
    prep_x<T, K, I, TIN, TOUT, ACC>();
    const size_t        sm = smem ? smem : ps.smem;
    const XformArgs<T>* pa = ps.dev.template as<XformArgs<T>>();
    if (eng == 1)
    {
        if (plan >= 0 && ps.tr[plan]->fd.M == kXformStaticM)
        {
            const void*     fn   = (const void*)k_xform_rc<T, K, I, TIN, TOUT, ACC, kXformStaticM>;
            const long long grid = std::min<long long>(sg.total, resident_ctas(fn, threads, sm));
            k_xform_rc<T, K, I, TIN, TOUT, ACC, kXformStaticM><<<(unsigned)grid, threads, sm, s>>>(
                sg.as<DstSeg>(), sg.pre(), sg.n, sg.total, DstSeg{}, ps.tr[plan]->hargs[I]);
            FPB_CHECK_LAUNCH();
            return;
        }
        const void*     fn   = (const void*)k_b_xform<T, K, I, TIN, TOUT, ACC, 1>;
        const long long grid = std::min<long long>(sg.total, resident_ctas(fn, threads, sm));
        k_b_xform<T, K, I, TIN, TOUT, ACC, 1><<<(unsigned)grid, threads, sm, s>>>(
            sg.as<DstSeg>(), sg.pre(), sg.n, sg.total, pa, DstSeg{}, XformArgs<T>{});
        FPB_CHECK_LAUNCH();
        return;
    }
    const long long grid = std::min<long long>(sg.total, (long long)sm_count() * tm.dst_blocks_per_sm);
    if (plan >= 0)
        k_b_xform<T, K, I, TIN, TOUT, ACC, 0, true><<<(unsigned)grid, tm.dst_threads, sm, s>>>(
            sg.as<DstSeg>(), sg.pre(), sg.n, sg.total, nullptr, DstSeg{}, ps.tr[plan]->hargs[I]);
    else
        k_b_xform<T, K, I, TIN, TOUT, ACC, 0><<<(unsigned)grid, tm.dst_threads, sm, s>>>(
            sg.as<DstSeg>(), sg.pre(), sg.n, sg.total, pa, DstSeg{}, XformArgs<T>{});
    FPB_CHECK_LAUNCH();
}

// DD and DN are their own inverses (the same kernel path); ND has a distinct inverse.
template <typename T, typename TIN, typename TOUT, bool ACC>
void launch_x(const XList& L, bool inverse, const PlanSet<T>& ps, const BatchTiming& tm, cudaStream_t s)
{
    for (auto& part : L.parts)
    {
        const int e = part.eng, th = part.threads, p = part.plan;
        switch (part.kind)
        {
            case K_DD: launch_x1<T, K_DD, 0, TIN, TOUT, ACC>(part.seg, ps, tm, s, part.smem, e, th, p); break;
            case K_DN: launch_x1<T, K_DN, 0, TIN, TOUT, ACC>(part.seg, ps, tm, s, part.smem, e, th, p); break;
            default:
                if (inverse) launch_x1<T, K_ND, 1, TIN, TOUT, ACC>(part.seg, ps, tm, s, part.smem, e, th, p);
                else launch_x1<T, K_ND, 0, TIN, TOUT, ACC>(part.seg, ps, tm, s, part.smem, e, th, p);
        }
    }
}

template <typename T, typename TIN, typename TOUT, bool ACC> void prep_x_all()
{
    prep_x<T, K_DD, 0, TIN, TOUT, ACC>();
    prep_x<T, K_DN, 0, TIN, TOUT, ACC>();
    prep_x<T, K_ND, 0, TIN, TOUT, ACC>();
    prep_x<T, K_ND, 1, TIN, TOUT, ACC>();
}

}  // namespace

template <typename TS> class BatchImpl final : public BatchBase
{
public:
    BatchImpl(const std::vector<BatchProblemDesc>& probs);
    ~BatchImpl() override
    {
        if (graph_) cudaGraphExecDestroy(graph_);
        if (irgraph_) cudaGraphExecDestroy(irgraph_);
        if (irhost_) cudaFreeHost(irhost_);
    }
    void solve(double* const* fields, const double* const* ghosts, int steps, cudaStream_t s) override;
    void solve_graph(double* const* fields, const double* const* ghosts, int steps, cudaStream_t s) override;
    void residuals(const double* const* u, const double* const* rhs, const double* const* ghosts, cudaStream_t s,
                   double* out) override;
    int           n_problems() const override { return (int)prob_.size(); }
    int           n_domains() const override { return (int)dom_.size(); }
    const Domain& domain(int g) const override { return dom_[g].d; }
    BatchTiming   timing() const override { return tm_; }
    void          autotune(cudaStream_t s) override;
    long long     graph_kernels() const override { return graph_kernels_; }
    int           refine(double* const* fields, const double* const* ghosts, double rel_tol, int max_refine,
                         cudaStream_t s, double* rel_change, BatchBase* first, bool defer) override;
    void          refine_result(int* steps, double* rel_change) override;
    void          solve_assembled(const double* const* in, double* const* out, cudaStream_t s) override;
    void          prepare_assembled(const double* const* in, double* const* out) override;
    long long     assembled_generation() const override { return ext_gen_; }

private:
    struct Dom
    {
        Domain    d;
        int       prob = 0, role = 0;  // role 0: root, 1: leaf
        int       leaf_face = -1;      // leaf: its face toward the root; root: -1
        int       root_face = -1;      // leaf: the root's face it is attached to
        int       plan = 0, tab = 0, kind = K_DD;
        long long off  = 0;            // element offset in W / X / fs / u / r
    };
    struct Prob
    {
        int    root = 0, g0 = 0, nd = 0;
        int    xe[2] = {-1, -1}, ye[2] = {-1, -1};  // leaves (global index) on the x / y edges, in edge order
        int    nxe = 0, nye = 0;
        BIface F{};
        DevBuf mem;  // spectral vectors and interface work (doubles)
        DevBuf rinv;
        DevBuf K;    // root inverse in the 2D basis (problems with both x- and y-edges)
        DevBuf part; // partial sums of the interface's dense products
    };

    void   build_spectral();
    void   build_static_lists();
    void   build_chase_lists();
    void   chase_run(const Segments& lc, const Segments& red, cudaStream_t s);
    void   inner(const XList& dst_in, const XList& dst_out, bool acc, cudaStream_t s, bool inv64 = false);
    void   first_inner(cudaStream_t s);
    void   build_plans64();
    const double* basis_col(int kind, int n, int j);
    bool   build_edge_mv(const std::vector<DstSeg>& segs, const std::vector<int>& ns, Segments& out);
    void   edge_mv(const Segments& l, cudaStream_t s);
    void   set_user_lists(double* const* fields, const double* const* ghosts, int steps);
    ResSeg res_seg(size_t g, double* r, const double* fs, const double* const* u_user);
    void   run(int steps, cudaStream_t s);
    void   drop_graphs();
    void   build_ir_graph(double rel_tol, int max_refine, BatchBase* first, const double* const* fi,
                          double* const* fo);
    int    ir_outcome(double* rel_change, long long runs);

    std::vector<DevBuf>                       eig_keep_;  // eigenvalue arrays referenced by BIface
    std::vector<Dom>                          dom_;
    std::vector<Prob>                         prob_;
    long long                                 cells_ = 0;
    PlanSet<TS>                               plans_;
    PlanSet<double>                           eplans_;  // FP64 DSTs of edge vectors (length nx of roots)
    // FP32 storage: FP64 plans of the same (family, length) at the same indices as plans_, for the first inner
    // solve's inverse transform, and the list writing its output into the iterate
    PlanSet<double>                           plans64_;
    XList                                     dst_out_u64_;
    BatchTiming                               tm64_;
    std::map<std::pair<int, double>, int>     tab_index_;
    std::vector<std::unique_ptr<DevRect<double>>> tabs_;  // chase tables (FP64 in both storage precisions)
    std::vector<DevBuf>                           tab_back_;  // the back substitution's copy of each cc
    DevBuf                                    tabs_dev_;
    DevBuf                                    W_, X_, fs_, r_, chs_;  // work, chase out, IR, chase scratch
    DevBuf                                    edge_;  // bY, gYp, sYp, yYp per y-edge (nx each), per problem
    std::vector<ChaseSeg<TS>>                 chase1_leaf_, chase1_root_, chase2_all_;
    Segments                                  l1_lc_, l1_red_, r1_lc_, r1_red_, a2_lc_, a2_red_;
    Segments                                  leaf_rows_, leaf_cols_, root_rows_, root_cols_;
    Segments                                  edst_g_, edst_out_;         // FP64 edge DSTs
    Segments                                  edge_mv_g_, edge_mv_o_;     // the same as dense products
    bool                                      mv_g_ = false, mv_o_ = false;
    std::map<int, DevBuf>                     edge_tab_;                  // DST-I matrices by length
    Segments                                  ifk_, ifym_, ifrow_, ifkw_;  // interface work lists
    Segments                                  ifyyp_, ifyxp_;              // partial-product blocks
    std::vector<DstSeg>                       dst_W_in_rec_, dst_X_out_rec_;
    std::vector<int>                          dst_kinds_;
    XList                                     dst_fs_, dst_r_, dst_out_u_, dst_out_r_, dst_user_in_, dst_user_out_;
    Segments                                  res_, asm_user_;
    Segments                                  addn_;  // u += r with norms (adaptive refinement)
    DevBuf                                    addp_;
    std::map<std::tuple<int, int, int>, DevBuf> basis_;  // y-basis column tables (family, n, column)
    std::vector<const double*>                ext_in_;     // solve_assembled: last pointer sets and lists
    std::vector<double*>                      ext_out_;
    XList                                     ext_in_list_, ext_out_list_;
    std::vector<double*>                      user_ptrs_;
    std::vector<const double*>                user_ghosts_;
    int                                       user_steps_ = -1;
    BatchTiming                               tm_;
    cudaGraphExec_t                           graph_         = nullptr;
    long long                                 graph_kernels_ = 0;
    long long                                 ext_gen_       = 0;  // rebuilds of ext_in_list_ / ext_out_list_
    // refinement graph (refine with max_refine > 1) and its key
    cudaGraphExec_t                           irgraph_  = nullptr;
    const BatchBase*                          irfirst_  = nullptr;
    int                                       irmax_    = 0;
    double                                    irtol_    = 0;
    long long                                 irgen_    = -1;
    long long                                 ir_pro_   = 0, ir_body_ = 0;  // kernels before / in the loop
    long long                                 ir_pending_ = 0;              // deferred runs not yet reported
    DevBuf                                    irst_;                        // IrState
    IrState*                                  irhost_ = nullptr;            // pinned copy of it after each run
    int                                       last_steps_  = 0;             // outcome of the last refinement
    double                                    last_change_ = 0;
};

template <typename TS> BatchImpl<TS>::BatchImpl(const std::vector<BatchProblemDesc>& probs)
{
    eplans_.stage_only = true;  // one launch covers edge rows of every length (one CTA shape)
    if (probs.empty()) throw Error(1, "empty batch");
    for (size_t p = 0; p < probs.size(); ++p)
    {
        const auto& P  = probs[p];
        const int   nd = (int)P.doms.size();
        if (nd <= 0) throw Error(1, "problem " + std::to_string(p) + " has no domains");
        Tree t = build_tree(nd, P.conns, -1);
        Prob pr;
        pr.g0   = (int)dom_.size();
        pr.nd   = nd;
        pr.root = pr.g0 + t.root;
        for (int d = 0; d < nd; ++d)
        {
            Dom D;
            D.d    = P.doms[d];
            D.prob = (int)p;
            const Domain& q = D.d;
            if (q.nx % kChunk != 0 || q.nx < 2 * kChunk)
                throw Error(3, "batched solve needs nx a multiple of 32 and >= 64 in every subdomain");
            if (q.ny < 2) throw Error(1, "each subdomain needs at least 2 cells per direction");
            auto dl = [](int b) { return b == BC_DIRICHLET || b == BC_ADJACENTED; };
            for (int f = 0; f < 4; ++f)
                if (q.bc[f] != BC_DIRICHLET && q.bc[f] != BC_ADJACENTED && q.bc[f] != BC_NEUMANN)
                    throw Error(3, "spectral solve supports Dirichlet and Neumann outer faces only");
            D.role = d == t.root ? 0 : 1;
            if (D.role == 0)
            {
                for (int f = 0; f < 4; ++f)
                    if (!dl(q.bc[f])) throw Error(3, "spectral solve needs Dirichlet faces on the root subdomain");
            }
            else
            {
                if (!t.children[d].empty() || t.parent[d].second != t.root)
                    throw Error(3, "spectral solve needs every subdomain attached to the root (depth-1 tree)");
                D.leaf_face = t.parent[d].first;
                D.root_face = D.leaf_face ^ 1;
                // the leaf's faces along the interface carry the root's transform basis
                const int a0 = D.leaf_face < 2 ? YNEG : XNEG;
                if (!dl(q.bc[a0]) || !dl(q.bc[a0 + 1]))
                    throw Error(3, "spectral solve needs Dirichlet faces on a leaf's sides along the interface");
            }
            D.kind = kind_of(q.bc[YNEG], q.bc[YPOS]);
            D.off = cells_;
            cells_ += q.cells();
            dom_.push_back(D);
        }
        for (auto& c : t.children[t.root])
        {
            const int face = c.first, g = pr.g0 + c.second;
            const Domain& R = dom_[pr.root].d;
            const Domain& L = dom_[g].d;
            if (face < 2)
            {
                if (L.ny != R.ny || L.hy != R.hy) throw Error(1, "x-connected subdomains must share ny and hy");
                pr.xe[pr.nxe++] = g;
            }
            else
            {
                if (L.nx != R.nx || L.hx != R.hx) throw Error(1, "y-connected subdomains must share nx and hx");
                pr.ye[pr.nye++] = g;
            }
        }
        prob_.push_back(std::move(pr));
    }
    // separator-factor rows each shared table needs: the largest P of the subdomains using it
    std::map<std::pair<int, double>, int> rows_needed;
    auto table_key = [](const Dom& D) {
        int bcd[4];
        for (int f = 0; f < 4; ++f) bcd[f] = D.d.bc[f] == BC_ADJACENTED ? BC_DIRICHLET : D.d.bc[f];
        const int sig = bcd[0] + 4 * bcd[1] + 16 * bcd[2] + 64 * bcd[3];
        return std::make_pair(D.d.ny * 256 + sig, D.d.hx * D.d.hx / D.d.hy / D.d.hy);
    };
    for (auto& D : dom_)
    {
        int& r = rows_needed[table_key(D)];
        r      = std::max(r, D.d.nx / kChunk);
    }
    for (auto& D : dom_)
    {
        D.plan = plans_.get(D.kind, D.d.ny);
        // chase tables depend on (ny, hx^2/hy^2, y family, x- / x+ Neumann)
        int bcd[4];
        for (int f = 0; f < 4; ++f) bcd[f] = D.d.bc[f] == BC_ADJACENTED ? BC_DIRICHLET : D.d.bc[f];
        const double r   = D.d.hx * D.d.hx / D.d.hy / D.d.hy;
        const int    sig = bcd[0] + 4 * bcd[1] + 16 * bcd[2] + 64 * bcd[3];
        auto         key = std::make_pair(D.d.ny * 256 + sig, r);
        auto         it  = tab_index_.find(key);
        if (it == tab_index_.end())
        {
            tabs_.emplace_back(new DevRect<double>(2 * kChunk, D.d.ny, D.d.hx, D.d.hy, bcd, rows_needed[key], false));
            it = tab_index_.emplace(key, (int)tabs_.size() - 1).first;
        }
        D.tab = it->second;
    }
    plans_.finish();
    std::vector<ChaseTabDev> tv;
    for (auto& t : tabs_)
    {
        tab_back_.emplace_back(t->cc.bytes());
        FPB_CUDA(cudaMemcpy(tab_back_.back().get(), t->cc.get(), t->cc.bytes(), cudaMemcpyDeviceToDevice));
        tv.push_back({t->cc.as<double>(), t->cg.as<double>(), t->chh.as<double>(), t->cends.as<double>(),
                      t->dsep.as<double>(), t->end_neumann ? 1 : 0, t->sep_cp.as<double>(), t->sep_iden.as<double>(),
                      tab_back_.back().as<double>()});
    }
    tabs_dev_ = upload(tv);
    W_.alloc((size_t)cells_ * sizeof(TS));
    X_.alloc((size_t)cells_ * sizeof(TS));
    long long sep = 0;
    for (auto& D : dom_) sep += (long long)(D.d.nx / kChunk) * D.d.ny * 4;
    chs_.alloc((size_t)sep * sizeof(double));
    build_spectral();
    build_static_lists();
    prep_x_all<TS, double, TS, false>();
    prep_x_all<TS, TS, double, false>();
    prep_x_all<TS, TS, double, true>();
    prep_x_all<TS, TS, TS, false>();
    prep_x<double, K_DD, 0, double, double, false>();
}

// Closed-form spectral responses, interface inverses and the reduced cross systems.
template <typename TS> void BatchImpl<TS>::build_spectral()
{
    // eigenvalues (cal_lambda - 2, the reference's own formula) per distinct length
    std::map<int, DevBuf> eig;
    auto eig_of = [&](int n) -> const double* {
        auto it = eig.find(n);
        if (it == eig.end())
        {
            std::vector<double> l = cal_lambda(n, BC_DIRICHLET, BC_DIRICHLET);
            for (auto& v : l) v -= 2.0;
            it = eig.emplace(n, upload(l)).first;
        }
        return it->second.template as<double>();
    };
    // Per problem: doubles laid out as sig[2](ny) sigp[2](nx) gX/zX/yX/bX/bX2 (2 ny each) gY/rhsY/yY/sY
    // (2 nx each), G blocks (ny * 4), H blocks (nx * 4), invxx (ny * 4), invyy (nx * 4)
    std::vector<GreenReq>  greq;
    std::vector<long long> gcnt;
    std::vector<EndReq>    ereq;
    std::vector<long long> ecnt;
    struct Host
    {
        std::vector<double> G, H, sig, sigp;
    };
    for (auto& pr : prob_)
    {
        const Domain& R  = dom_[pr.root].d;
        const int     nx = R.nx, ny = R.ny;
        const size_t  nd = 2 * ny + 2 * nx + 5 * 2 * ny + 4 * 2 * nx + 4 * ny + 4 * nx + 4 * ny + 4 * nx + 4 * ny + 4 * nx;
        pr.mem.alloc(nd * sizeof(double));
        FPB_CUDA(cudaMemset(pr.mem.get(), 0, nd * sizeof(double)));
        double* b = pr.mem.template as<double>();
        BIface& F = pr.F;
        F.nx = nx;
        F.ny = ny;
        F.nxe = pr.nxe;
        F.nye = pr.nye;
        F.r   = R.hx * R.hx / R.hy / R.hy;
        F.alpha = eig_of(nx);
        F.beta  = eig_of(ny);
        double* sig  = b;
        double* sigp = sig + 2 * ny;
        double* v    = sigp + 2 * nx;
        F.gX  = v;
        F.zX  = v + 2 * ny;
        F.yX  = v + 4 * ny;
        F.bX  = v + 6 * ny;
        F.bX2 = v + 8 * ny;
        v += 10 * ny;
        F.gY   = v;
        F.rhsY = v + 2 * nx;
        F.yY   = v + 4 * nx;
        F.sY   = v + 6 * nx;
        v += 8 * nx;
        double* Gd = v;  // G[(e*2+e2)*ny + k]
        double* Hd = v + 4 * ny;
        double* ix = Hd + 4 * nx;
        double* iy = ix + 4 * ny;
        F.invxx    = ix;
        F.invyy    = iy;
        F.vxy      = iy + 4 * nx;
        F.wxy      = F.vxy + 4 * ny;
        for (int e = 0; e < pr.nxe; ++e)
        {
            const Dom& L = dom_[pr.xe[e]];
            F.ie[e]      = L.root_face == XNEG ? 0 : nx - 1;
            F.sig[e]     = sig + e * ny;
            // the leaf's response at its interface row: Dirichlet tridiagonal with the leaf's own x- / x+
            // Neumann ends, per y-mode of the shared (DD) basis
            eig_keep_.push_back(upload(x_diag(ny, L.d.hx, L.d.hy, BC_DIRICHLET, BC_DIRICHLET)));
            ereq.push_back({L.d.nx, L.leaf_face == XNEG ? 1 : 0, L.d.bc[XNEG] == BC_NEUMANN ? 1 : 0,
                            L.d.bc[XPOS] == BC_NEUMANN ? 1 : 0, ny, eig_keep_.back().template as<double>(),
                            sig + e * ny});
            ecnt.push_back(ny);
            for (int e2 = 0; e2 < pr.nxe; ++e2)
            {
                const Dom& L2 = dom_[pr.xe[e2]];
                const int  i2 = L2.root_face == XNEG ? 0 : nx - 1;
                greq.push_back({nx, F.ie[e], i2, ny, F.alpha, F.beta, F.r, Gd + (e * 2 + e2) * ny});
                gcnt.push_back(ny);
            }
        }
        for (int Y = 0; Y < pr.nye; ++Y)
        {
            const Dom& L = dom_[pr.ye[Y]];
            F.jy[Y]      = L.root_face == YNEG ? 0 : ny - 1;
            F.sigp[Y]    = sigp + Y * nx;
            const int jl = L.leaf_face == YNEG ? 0 : L.d.ny - 1;
            // sig'_m = sum_k psi_k(jl)^2 / (alpha_m + r_l beta^l_k): sum index over the leaf's ny
            const double rl = L.d.hx * L.d.hx / L.d.hy / L.d.hy;
            {
                // eig_a = r_l * beta^l (the leaf's own y family), so that k_green's form eig_a[k] + 1 * alpha_m
                // applies; weights: the squared y-basis value at the interface row
                const int yn = L.d.bc[YNEG] == BC_ADJACENTED ? BC_DIRICHLET : L.d.bc[YNEG];
                const int yp = L.d.bc[YPOS] == BC_ADJACENTED ? BC_DIRICHLET : L.d.bc[YPOS];
                std::vector<double> l = cal_lambda(L.d.ny, yn, yp);
                for (auto& q : l) q = rl * (q - 2.0);
                eig_keep_.push_back(upload(l));
                const double* eg = eig_keep_.back().template as<double>();
                const double* wt = nullptr;
                if (L.kind != K_DD)
                {
                    const double*       tab = basis_col(L.kind, L.d.ny, jl);
                    std::vector<double> w(L.d.ny);
                    FPB_CUDA(cudaMemcpy(w.data(), tab, w.size() * 8, cudaMemcpyDeviceToHost));
                    for (auto& q : w) q = q * q;
                    eig_keep_.push_back(upload(w));
                    wt = eig_keep_.back().template as<double>();
                }
                greq.push_back({L.d.ny, jl, jl, nx, eg, F.alpha, 1.0, sigp + Y * nx, wt});
            }
            gcnt.push_back(nx);
            for (int Y2 = 0; Y2 < pr.nye; ++Y2)
            {
                const Dom& L2 = dom_[pr.ye[Y2]];
                const int  j2 = L2.root_face == YNEG ? 0 : ny - 1;
                std::vector<double> l = cal_lambda(ny, BC_DIRICHLET, BC_DIRICHLET);
                for (auto& q : l) q = F.r * (q - 2.0);
                eig_keep_.push_back(upload(l));
                greq.push_back({ny, F.jy[Y], j2, nx, eig_keep_.back().template as<double>(), F.alpha, 1.0,
                                Hd + (Y * 2 + Y2) * nx});
                gcnt.push_back(nx);
            }
        }
    }
    if (!greq.empty())
    {
        Segments g;
        g.set(greq, gcnt);
        k_green<<<grid_of(g.total * 32, 256), 256>>>(g.as<GreenReq>(), g.pre(), g.n);
        FPB_CHECK_LAUNCH();
        FPB_CUDA(cudaDeviceSynchronize());
    }
    if (!ereq.empty())
    {
        Segments g;
        g.set(ereq, ecnt);
        k_green_end<<<grid_of(g.total, 128), 128>>>(g.as<EndReq>(), g.pre(), g.n);
        FPB_CHECK_LAUNCH();
        FPB_CUDA(cudaDeviceSynchronize());
    }
    // interface inverses (host, tiny) and reduced cross systems (device)
    cublasHandle_t     cb = nullptr;
    cusolverDnHandle_t cs = nullptr;
    DevBuf             A, B, piv, info, work;
    for (auto& pr : prob_)
    {
        BIface&   F  = pr.F;
        const int nx = F.nx, ny = F.ny;
        double*   b  = pr.mem.template as<double>();
        double*   Gd = b + 2 * ny + 2 * nx + 10 * ny + 8 * nx;
        double*   Hd = Gd + 4 * ny;
        std::vector<double> G(4 * ny), H(4 * nx), sg(2 * ny), sp(2 * nx);
        FPB_CUDA(cudaMemcpy(G.data(), Gd, G.size() * 8, cudaMemcpyDeviceToHost));
        FPB_CUDA(cudaMemcpy(H.data(), Hd, H.size() * 8, cudaMemcpyDeviceToHost));
        FPB_CUDA(cudaMemcpy(sg.data(), b, sg.size() * 8, cudaMemcpyDeviceToHost));
        FPB_CUDA(cudaMemcpy(sp.data(), b + 2 * ny, sp.size() * 8, cudaMemcpyDeviceToHost));
        auto inv_blocks = [](int E, int n, const std::vector<double>& Gm, const std::vector<double>& s) {
            // M = I - G(e, e2) s_e2 per mode; returns row-major E x E inverses per mode
            std::vector<double> out((size_t)n * E * E, 0.0);
            for (int q = 0; q < n; ++q)
            {
                if (E == 1)
                {
                    out[q] = 1.0 / (1.0 - Gm[q] * s[q]);
                }
                else if (E == 2)
                {
                    const double a = 1.0 - Gm[0 * n + q] * s[q], bb = -Gm[1 * n + q] * s[n + q];
                    const double c = -Gm[2 * n + q] * s[q], d = 1.0 - Gm[3 * n + q] * s[n + q];
                    const double det = a * d - bb * c;
                    out[(size_t)q * 4 + 0] = d / det;
                    out[(size_t)q * 4 + 1] = -bb / det;
                    out[(size_t)q * 4 + 2] = -c / det;
                    out[(size_t)q * 4 + 3] = a / det;
                }
            }
            return out;
        };
        if (F.nxe > 0)
        {
            std::vector<double> ix = inv_blocks(F.nxe, ny, G, sg);
            FPB_CUDA(cudaMemcpy(const_cast<double*>(F.invxx), ix.data(), ix.size() * 8, cudaMemcpyHostToDevice));
        }
        if (F.nye > 0 && F.nxe == 0)
        {
            std::vector<double> iy = inv_blocks(F.nye, nx, H, sp);
            FPB_CUDA(cudaMemcpy(const_cast<double*>(F.invyy), iy.data(), iy.size() * 8, cudaMemcpyHostToDevice));
        }
        if (F.nxe > 0 && F.nye > 0)
        {
            const int nYp = F.nye * nx;
            F.yy_chunks   = (nYp + kIfChunkYY - 1) / kIfChunkYY;
            F.yx_chunks   = (nx + kIfChunkYX - 1) / kIfChunkYX;
            pr.part.alloc(((size_t)F.yy_chunks * nYp + (size_t)F.yx_chunks * 4 * ny) * 8);
            FPB_CUDA(cudaMemset(pr.part.get(), 0, pr.part.bytes()));
            F.part_yy = pr.part.template as<double>();
            F.part_yx = F.part_yy + (size_t)F.yy_chunks * nYp;
            pr.K.alloc((size_t)nx * ny * 8);
            F.K = pr.K.template as<double>();
            k_root_inverse<<<grid_of((long long)nx * ny, 256), 256>>>(F, pr.K.template as<double>());
            FPB_CHECK_LAUNCH();
            const int nY = F.nye * nx, nX = F.nxe * ny;
            if (!cb)
            {
                if (cublasCreate(&cb) != CUBLAS_STATUS_SUCCESS) throw Error(2, "cublasCreate failed");
                if (cusolverDnCreate(&cs) != CUSOLVER_STATUS_SUCCESS) throw Error(2, "cusolverDnCreate failed");
            }
            A.ensure((size_t)nY * nX * 8);
            B.ensure((size_t)nY * nX * 8);
            pr.rinv.alloc((size_t)nY * nY * 8);
            DevBuf Rm((size_t)nY * nY * 8);
            k_cross_AB<<<grid_of((long long)nY * nX, 256), 256>>>(F, A.as<double>(), B.as<double>());
            FPB_CHECK_LAUNCH();
            k_myy<<<grid_of((long long)nY * nY, 256), 256>>>(F, Hd, Rm.as<double>());
            FPB_CHECK_LAUNCH();
            const double m1 = -1.0, one = 1.0;
            if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, nY, nY, nX, &m1, A.as<double>(), nY, B.as<double>(), nX,
                            &one, Rm.as<double>(), nY) != CUBLAS_STATUS_SUCCESS)
                throw Error(2, "cublasDgemm failed");
            int lw = 0;
            if (cusolverDnDgetrf_bufferSize(cs, nY, nY, Rm.as<double>(), nY, &lw) != CUSOLVER_STATUS_SUCCESS)
                throw Error(2, "cusolverDnDgetrf_bufferSize failed");
            work.ensure((size_t)std::max(lw, 1) * 8);
            piv.ensure((size_t)nY * 4);
            info.ensure(4);
            if (cusolverDnDgetrf(cs, nY, nY, Rm.as<double>(), nY, work.as<double>(), piv.as<int>(), info.as<int>()) !=
                CUSOLVER_STATUS_SUCCESS)
                throw Error(2, "cusolverDnDgetrf failed");
            std::vector<double> I((size_t)nY * nY, 0.0);
            for (int q = 0; q < nY; ++q) I[(size_t)q * nY + q] = 1.0;
            FPB_CUDA(cudaMemcpy(pr.rinv.get(), I.data(), I.size() * 8, cudaMemcpyHostToDevice));
            if (cusolverDnDgetrs(cs, CUBLAS_OP_N, nY, nY, Rm.as<double>(), nY, piv.as<int>(), pr.rinv.template as<double>(), nY,
                                 info.as<int>()) != CUSOLVER_STATUS_SUCCESS)
                throw Error(2, "cusolverDnDgetrs failed");
            int hinfo = 0;
            FPB_CUDA(cudaMemcpy(&hinfo, info.get(), 4, cudaMemcpyDeviceToHost));
            if (hinfo != 0) throw Error(5, "singular reduced interface system");
            F.rinv = pr.rinv.template as<double>();
        }
    }
    FPB_CUDA(cudaDeviceSynchronize());
    if (cs) cusolverDnDestroy(cs);
    if (cb) cublasDestroy(cb);
    for (auto& kv : eig) eig_keep_.push_back(std::move(kv.second));  // alpha / beta stay referenced
}

// Column j of the forward y-transform matrix of `kind` at length n (every family is orthonormal with the
// transpose as inverse, so this is also row j of the inverse): the FP64 transform of the unit vector e_j.
// Null for DD, whose basis dst_basis() evaluates directly.
// The edge DSTs of one list as dense products (k_edge_dst_mv) when the matrices they read are small: the rows of
// each length grouped kEdgeMvRows at a time, every group reading its n x n matrix once. Returns false (the FFT
// form stays) when the matrices' reads would pass 64 MB, as for the many lengths of a large batch.
template <typename TS>
bool BatchImpl<TS>::build_edge_mv(const std::vector<DstSeg>& segs, const std::vector<int>& ns, Segments& out)
{
    std::map<int, std::vector<size_t>> by_n;
    for (size_t q = 0; q < segs.size(); ++q) by_n[ns[q]].push_back(q);
    long long bytes = 0;
    for (auto& kv : by_n)
        bytes += (long long)((kv.second.size() + kEdgeMvRows - 1) / kEdgeMvRows) * kv.first * kv.first * 8;
    if (segs.empty() || bytes > (64LL << 20)) return false;
    std::vector<EdgeMv>    recs;
    std::vector<long long> counts;
    const long double      pi = 3.141592653589793238462643383279502884L;
    for (auto& kv : by_n)
    {
        const int n = kv.first;
        if (!edge_tab_.count(n))
        {
            const double        sc = std::sqrt(2.0 / (n + 1));
            std::vector<double> T((size_t)n * n);
            for (int k = 0; k < n; ++k)
                for (int i = 0; i < n; ++i)
                {
                    const long long q = (long long)(k + 1) * (i + 1) % (2LL * (n + 1));
                    T[(size_t)k * n + i] = sc * (double)std::sin(pi * (long double)q / (long double)(n + 1));
                }
            edge_tab_[n] = upload(T);
        }
        for (size_t a = 0; a < kv.second.size(); a += kEdgeMvRows)
        {
            EdgeMv r{};
            r.T = edge_tab_[n].template as<double>();
            r.n = n;
            for (size_t b = a; b < kv.second.size() && b < a + kEdgeMvRows; ++b)
            {
                const DstSeg& d   = segs[kv.second[b]];
                r.in[r.rows]      = static_cast<const double*>(d.in);
                r.out[r.rows]     = static_cast<double*>(d.out);
                ++r.rows;
            }
            recs.push_back(r);
            counts.push_back(n);
        }
    }
    out.set(recs, counts);
    return true;
}

template <typename TS> void BatchImpl<TS>::edge_mv(const Segments& l, cudaStream_t s)
{
    k_edge_dst_mv<<<(unsigned)l.total, kEdgeMvThreads, 0, s>>>(l.as<EdgeMv>(), l.pre(), l.n);
    FPB_CHECK_LAUNCH();
}

template <typename TS> const double* BatchImpl<TS>::basis_col(int kind, int n, int j)
{
    auto key = std::make_tuple(kind, n, j);
    auto it  = basis_.find(key);
    if (it != basis_.end()) return it->second.template as<double>();
    if (kind == K_DD)  // the DST-I basis in closed form, as dst_basis (sin in long double)
    {
        const long double   pi = 3.141592653589793238462643383279502884L;
        const double        sc = std::sqrt(2.0 / (n + 1));
        std::vector<double> e(n);
        for (int k = 0; k < n; ++k)
        {
            const long long q = (long long)(k + 1) * (j + 1) % (2LL * (n + 1));
            e[k]              = sc * (double)std::sin(pi * (long double)q / (long double)(n + 1));
        }
        return (basis_[key] = upload(e)).template as<double>();
    }
    DevTransform<double> tr(kind, n);
    std::vector<double>  e(n, 0.0);
    e[j]      = 1.0;
    DevBuf in = upload(e);
    DevBuf out((size_t)n * 8);
    tr.run(in.as<double>(), out.as<double>(), 1, false, 0);
    FPB_CUDA(cudaDeviceSynchronize());
    return (basis_[key] = std::move(out)).template as<double>();
}

template <typename TS> void BatchImpl<TS>::build_static_lists()
{
    const int nP = (int)prob_.size();
    // per-problem y-edge vectors: bY, gYp, sYp, yYp (nx each) for up to 2 y-edges
    std::vector<long long> eoff(nP + 1, 0);
    for (int p = 0; p < nP; ++p) eoff[p + 1] = eoff[p] + (long long)8 * prob_[p].F.nx;
    edge_.alloc((size_t)std::max<long long>(eoff[nP], 1) * sizeof(double));
    FPB_CUDA(cudaMemset(edge_.get(), 0, (size_t)std::max<long long>(eoff[nP], 1) * sizeof(double)));
    auto ev = [&](int p, int Y, int which) {  // which: 0 bY, 1 gYp, 2 sYp, 3 yYp
        return edge_.as<double>() + eoff[p] + (long long)(Y * 4 + which) * prob_[p].F.nx;
    };
    TS*       W = W_.as<TS>();
    TS*       X = X_.as<TS>();
    // chase scratch offsets
    std::vector<long long> soff(dom_.size() + 1, 0);
    for (size_t g = 0; g < dom_.size(); ++g)
        soff[g + 1] = soff[g] + (long long)(dom_[g].d.nx / kChunk) * dom_[g].d.ny * 4;
    auto base_seg = [&](int g, const TS* in, TS* out) {
        ChaseSeg<TS> c{};
        const Dom&   D = dom_[g];
        const long long P = D.d.nx / kChunk;
        c.in   = in;
        c.out  = out;
        c.nx   = D.d.nx;
        c.ny   = D.d.ny;
        c.tab  = D.tab;
        c.zend = chs_.as<double>() + soff[g];
        c.bsep = c.zend + 2 * P * D.d.ny;
        c.work = c.bsep + P * D.d.ny;
        return c;
    };
    std::vector<ChaseSeg<TS>> l1, r1, a2;
    std::vector<RowReq<TS>>   lr, rr;
    std::vector<ColReq<TS>>   lc, rc;
    std::vector<DstSeg>       eg, eo;
    std::vector<int>          eg_n, eo_n;  // their row lengths
    std::vector<BIface>       fk, fy, fr, fw;
    std::vector<long long>    ck, cy, cr, cw, lrc, rrc, lcc, rcc;
    for (int p = 0; p < nP; ++p)
    {
        Prob&     pr = prob_[p];
        BIface&   F  = pr.F;
        const int gr = pr.root;
        const long long ro = dom_[gr].off;
        for (int e = 0; e < pr.nxe; ++e)
        {
            const int   g = pr.xe[e];
            const Dom&  L = dom_[g];
            const int   il = L.leaf_face == XNEG ? 0 : L.d.nx - 1;
            l1.push_back(base_seg(g, W + L.off, X + L.off));
            lr.push_back({X + L.off, L.d.ny, il, F.bX + e * F.ny, -1.0});
            rr.push_back({X + ro, F.ny, F.ie[e], F.gX + e * F.ny, 1.0});
            ChaseSeg<TS> c = base_seg(g, W + L.off, X + L.off);
            c.nrow         = 1;
            c.row_i[0]     = il;
            c.row_v[0]     = F.yX + e * F.ny;
            c.row_c[0]     = -1.0;
            a2.push_back(c);
        }
        for (int Y = 0; Y < pr.nye; ++Y)
        {
            const int  g  = pr.ye[Y];
            const Dom& L  = dom_[g];
            const int  jl = L.leaf_face == YNEG ? 0 : L.d.ny - 1;
            l1.push_back(base_seg(g, W + L.off, X + L.off));
            lc.push_back({X + L.off, L.d.nx, L.d.ny, jl, ev(p, Y, 0), -1.0, basis_col(L.kind, L.d.ny, jl)});
            rc.push_back({X + ro, F.nx, F.ny, F.jy[Y], ev(p, Y, 1), 1.0, basis_col(K_DD, F.ny, F.jy[Y])});
            eg.push_back({ev(p, Y, 1), F.gY + Y * F.nx, 1, eplans_.get(K_DD, F.nx)});
            eo.push_back({F.sY + Y * F.nx, ev(p, Y, 2), 1, eplans_.get(K_DD, F.nx)});
            eo.push_back({F.yY + Y * F.nx, ev(p, Y, 3), 1, eplans_.get(K_DD, F.nx)});
            eg_n.push_back(F.nx);
            eo_n.push_back(F.nx);
            eo_n.push_back(F.nx);
            ChaseSeg<TS> c = base_seg(g, W + L.off, X + L.off);
            c.ncol         = 1;
            c.col_j[0]     = jl;
            c.col_s[0]     = ev(p, Y, 3);
            c.col_tab[0]   = basis_col(L.kind, L.d.ny, jl);
            c.col_c[0]     = -1.0;
            a2.push_back(c);
        }
        // root: first chase with the b' terms, second with b' + S y
        ChaseSeg<TS> c1 = base_seg(gr, W + ro, X + ro), c2 = c1;
        for (int e = 0; e < pr.nxe; ++e)
        {
            c1.row_i[c1.nrow] = F.ie[e];
            c1.row_v[c1.nrow] = F.bX + e * F.ny;
            c1.row_c[c1.nrow++] = 1.0;
            c2.row_i[c2.nrow] = F.ie[e];
            c2.row_v[c2.nrow] = F.bX2 + e * F.ny;
            c2.row_c[c2.nrow++] = 1.0;
        }
        for (int Y = 0; Y < pr.nye; ++Y)
        {
            c1.col_j[c1.ncol] = F.jy[Y];
            c1.col_s[c1.ncol] = ev(p, Y, 0);
            c1.col_c[c1.ncol++] = 1.0;
            c2.col_j[c2.ncol] = F.jy[Y];
            c2.col_s[c2.ncol] = ev(p, Y, 0);
            c2.col_c[c2.ncol++] = 1.0;
            c2.col_j[c2.ncol] = F.jy[Y];
            c2.col_s[c2.ncol] = ev(p, Y, 2);
            c2.col_c[c2.ncol++] = 1.0;
        }
        if (pr.nxe + pr.nye > 0) r1.push_back(c1);
        a2.push_back(c2);
        if (pr.nxe > 0)
        {
            fk.push_back(F);
            ck.push_back(F.ny);
            fw.push_back(F);
            cw.push_back(F.ny);
        }
        if (pr.nye > 0)
        {
            fy.push_back(F);
            cy.push_back((long long)F.nye * F.nx);
            fr.push_back(F);
            cr.push_back((long long)F.nye * F.nx);
        }
    }
    eplans_.finish();
    chase1_leaf_ = l1;
    chase1_root_ = r1;
    chase2_all_  = a2;
    build_chase_lists();
    for (auto& q : lr) lrc.push_back(q.ny);
    for (auto& q : rr) rrc.push_back(q.ny);
    for (auto& q : lc) lcc.push_back(q.nx);
    for (auto& q : rc) rcc.push_back(q.nx);
    leaf_rows_.set(lr, lrc);
    root_rows_.set(rr, rrc);
    leaf_cols_.set(lc, lcc);
    root_cols_.set(rc, rcc);
    std::vector<long long> one_e(eg.size(), 1), one_o(eo.size(), 1);
    edst_g_.set(eg, one_e);
    edst_out_.set(eo, one_o);
    mv_g_ = build_edge_mv(eg, eg_n, edge_mv_g_);
    mv_o_ = build_edge_mv(eo, eo_n, edge_mv_o_);
    {
        std::vector<BIface>    py, px;
        std::vector<long long> cy2, cx2;
        for (auto& pr : prob_)
            if (pr.F.nxe > 0 && pr.F.nye > 0)
            {
                const BIface& F = pr.F;
                py.push_back(F);
                cy2.push_back((long long)((F.nye * F.nx + kIfTile - 1) / kIfTile) * F.yy_chunks);
                px.push_back(F);
                cx2.push_back((long long)((F.ny + kIfTile - 1) / kIfTile) * F.yx_chunks);
            }
        ifyyp_.set(py, cy2);
        ifyxp_.set(px, cx2);
    }
    ifk_.set(fk, ck);
    ifkw_.set(fw, cw);
    ifym_.set(fy, cy);
    ifrow_.set(fr, cr);
    // transform lists over all subdomains between internal buffers (split by family where used)
    std::vector<DstSeg> dfs, dou;
    std::vector<int>    kinds;
    for (auto& D : dom_)
    {
        kinds.push_back(D.kind);
        dfs.push_back({nullptr, W + D.off, D.d.nx, D.plan});
        dou.push_back({X + D.off, nullptr, D.d.nx, D.plan});
    }
    dst_W_in_rec_  = dfs;
    dst_X_out_rec_ = dou;
    dst_kinds_     = kinds;
}

template <typename TS> void BatchImpl<TS>::build_chase_lists()
{
    const int bt = tm_.chase_threads;
    auto mk = [&](const std::vector<ChaseSeg<TS>>& v, Segments& lc, Segments& red) {
        std::vector<long long> a, b;
        for (auto& c : v)
        {
            a.push_back(((long long)(c.nx / kChunk) * c.ny + bt - 1) / bt);
            b.push_back((c.ny + 31) / 32);
        }
        lc.set(v, a);
        red.set(v, b);
    };
    mk(chase1_leaf_, l1_lc_, l1_red_);
    mk(chase1_root_, r1_lc_, r1_red_);
    mk(chase2_all_, a2_lc_, a2_red_);
}

template <typename TS> void BatchImpl<TS>::chase_run(const Segments& lc, const Segments& red, cudaStream_t s)
{
    if (lc.n == 0) return;
    const ChaseTabDev* tabs = tabs_dev_.as<ChaseTabDev>();
    k_b_chase_local<TS><<<(unsigned)lc.total, tm_.chase_threads, 0, s>>>(lc.as<ChaseSeg<TS>>(), lc.pre(), lc.n, tabs);
    FPB_CHECK_LAUNCH();
    k_b_chase_reduced<TS><<<(unsigned)red.total, 32 * kRedWarps, 0, s>>>(red.as<ChaseSeg<TS>>(), red.pre(), red.n, tabs);
    FPB_CHECK_LAUNCH();
    k_b_chase_correct<TS><<<(unsigned)lc.total, tm_.chase_threads, 0, s>>>(lc.as<ChaseSeg<TS>>(), lc.pre(), lc.n, tabs);
    FPB_CHECK_LAUNCH();
}

// One inner solve: dst_in (FP64 rows -> W), ..., X -> dst_out (FP64 rows; += when acc).
template <typename TS>
void BatchImpl<TS>::inner(const XList& dst_in, const XList& dst_out, bool acc, cudaStream_t s, bool inv64)
{
    launch_x<TS, double, TS, false>(dst_in, false, plans_, tm_, s);
    chase_run(l1_lc_, l1_red_, s);
    if (leaf_rows_.n)
    {
        k_b_rowcopy<TS><<<grid_of(leaf_rows_.total, 256), 256, 0, s>>>(leaf_rows_.as<RowReq<TS>>(), leaf_rows_.pre(),
                                                                    leaf_rows_.n);
        FPB_CHECK_LAUNCH();
    }
    if (leaf_cols_.n)
    {
        k_b_colvals<TS><<<grid_of(leaf_cols_.total * 32, 256), 256, 0, s>>>(leaf_cols_.as<ColReq<TS>>(),
                                                                         leaf_cols_.pre(), leaf_cols_.n);
        FPB_CHECK_LAUNCH();
    }
    chase_run(r1_lc_, r1_red_, s);
    if (root_rows_.n)
    {
        k_b_rowcopy<TS><<<grid_of(root_rows_.total, 256), 256, 0, s>>>(root_rows_.as<RowReq<TS>>(), root_rows_.pre(),
                                                                    root_rows_.n);
        FPB_CHECK_LAUNCH();
    }
    if (root_cols_.n)
    {
        k_b_colvals<TS><<<grid_of(root_cols_.total * 32, 256), 256, 0, s>>>(root_cols_.as<ColReq<TS>>(),
                                                                         root_cols_.pre(), root_cols_.n);
        FPB_CHECK_LAUNCH();
    }
    if (mv_g_) edge_mv(edge_mv_g_, s);
    else launch_x1<double, K_DD, 0, double, double, false>(edst_g_, eplans_, tm_, s);
    if (ifk_.n)
    {
        k_if_zx<<<grid_of(ifk_.total, 128), 128, 0, s>>>(ifk_.as<BIface>(), ifk_.pre(), ifk_.n);
        FPB_CHECK_LAUNCH();
    }
    if (ifym_.n)
    {
        k_if_rhsy<<<grid_of(ifym_.total * 32, 256), 256, 0, s>>>(ifym_.as<BIface>(), ifym_.pre(), ifym_.n);
        FPB_CHECK_LAUNCH();
        if (ifyyp_.n)
        {
            k_if_yy_part<<<(unsigned)ifyyp_.total, 256, 0, s>>>(ifyyp_.as<BIface>(), ifyyp_.pre(), ifyyp_.n);
            FPB_CHECK_LAUNCH();
        }
        k_if_yy<<<grid_of(ifrow_.total, 128), 128, 0, s>>>(ifrow_.as<BIface>(), ifrow_.pre(), ifrow_.n);
        FPB_CHECK_LAUNCH();
    }
    if (ifkw_.n)
    {
        if (ifyxp_.n)
        {
            k_if_yx_part<<<(unsigned)ifyxp_.total, 256, 0, s>>>(ifyxp_.as<BIface>(), ifyxp_.pre(), ifyxp_.n);
            FPB_CHECK_LAUNCH();
        }
        k_if_yx<<<grid_of(ifkw_.total, 128), 128, 0, s>>>(ifkw_.as<BIface>(), ifkw_.pre(), ifkw_.n);
        FPB_CHECK_LAUNCH();
    }
    if (mv_o_) edge_mv(edge_mv_o_, s);
    else launch_x1<double, K_DD, 0, double, double, false>(edst_out_, eplans_, tm_, s);
    chase_run(a2_lc_, a2_red_, s);
    if constexpr (std::is_same<TS, float>::value)
        if (inv64)
        {
            launch_x<double, TS, double, false>(dst_out, true, plans64_, tm64_, s);
            return;
        }
    if (acc) launch_x<TS, TS, double, true>(dst_out, true, plans_, tm_, s);
    else launch_x<TS, TS, double, false>(dst_out, true, plans_, tm_, s);
}

// The first inner solve of a refinement (right-hand sides in fs, solution written into the iterate). With
// FP32 storage its inverse transform runs in FP64 arithmetic on the FP32 chase output: the DST-I's folding
// algorithm sums ~n/2 FFT outputs into the odd coefficients, so an FP32 inverse leaves a random-walk error
// (~3e-6 at n = 2048) that the first correction contracts only to ~6e-10; with the FP64 inverse the first
// solve is ~8e-8 from the answer and one FP32 correction reaches ~3e-13.
template <typename TS> void BatchImpl<TS>::first_inner(cudaStream_t s)
{
    if (std::is_same<TS, float>::value) inner(dst_fs_, dst_out_u64_, false, s, true);
    else inner(dst_fs_, dst_out_u_, false, s);
}

template <typename TS> void BatchImpl<TS>::build_plans64()
{
    if (!std::is_same<TS, float>::value || !plans64_.tr.empty()) return;
    for (auto& D : dom_)
        if (plans64_.get(D.kind, D.d.ny) != D.plan) throw Error(2, "FP64 plan indices differ from the FP32 plans");
    plans64_.finish();
    tm64_                   = tm_;
    tm64_.dst_threads       = 128;      // the FP64 batch's measured stage-engine shape
    tm64_.dst_blocks_per_sm = 1 << 20;  // one CTA per work item
}

template <typename TS>
void BatchImpl<TS>::set_user_lists(double* const* fields, const double* const* ghosts, int steps)
{
    const int nd = (int)dom_.size();
    std::vector<double*>       f(fields, fields + nd);
    std::vector<const double*> gh;
    if (ghosts) gh.assign(ghosts, ghosts + 4 * nd);
    if (f == user_ptrs_ && gh == user_ghosts_ && steps == user_steps_) return;
    drop_graphs();
    FPB_CUDA(cudaDeviceSynchronize());  // the lists below may still be read by queued work
    user_ptrs_   = f;
    user_ghosts_ = gh;
    user_steps_  = steps;
    const bool ir = steps > 0;
    if (ir && !fs_.get())
    {
        fs_.alloc((size_t)cells_ * 8);
        r_.alloc((size_t)cells_ * 8);
        // IR lists between internal buffers
        std::vector<DstSeg> a = dst_W_in_rec_, b = dst_W_in_rec_;
        for (size_t g = 0; g < dom_.size(); ++g)
        {
            a[g].in = fs_.as<double>() + dom_[g].off;
            b[g].in = r_.as<double>() + dom_[g].off;
        }
        dst_fs_.set(a, dst_kinds_, plans_);
        dst_r_.set(b, dst_kinds_, plans_);
        std::vector<DstSeg> d = dst_X_out_rec_;
        for (size_t g = 0; g < dom_.size(); ++g) d[g].out = r_.as<double>() + dom_[g].off;
        dst_out_r_.set(d, dst_kinds_, plans_);
        long long nb = 0;
        for (size_t g = 0; g < dom_.size(); ++g) nb += (dom_[g].d.cells() + kElemCells - 1) / kElemCells;
        addp_.alloc((size_t)2 * nb * 8);
    }
    if (ir)  // the iterate u lives in the caller's fields (their right-hand sides are in fs once assembled)
    {
        std::vector<DstSeg> c = dst_X_out_rec_;
        for (int g = 0; g < nd; ++g) c[g].out = f[g];
        dst_out_u_.set(c, dst_kinds_, plans_);
        if (std::is_same<TS, float>::value)
        {
            build_plans64();
            dst_out_u64_.set(c, dst_kinds_, plans64_);
        }
        const long long        nb = (long long)(addp_.bytes() / 16);
        std::vector<AddSeg>    ad;
        std::vector<long long> acn;
        long long              b0 = 0;
        for (int g = 0; g < nd; ++g)
        {
            const long long blocks = (dom_[g].d.cells() + kElemCells - 1) / kElemCells;
            ad.push_back({f[g], r_.as<double>() + dom_[g].off, dom_[g].d.cells(), addp_.as<double>() + b0,
                          addp_.as<double>() + nb + b0});
            acn.push_back(blocks);
            b0 += blocks;
        }
        addn_.set(ad, acn);
        std::vector<ResSeg>    rs;
        std::vector<long long> rc;
        for (int g = 0; g < nd; ++g) rs.push_back(res_seg(g, r_.as<double>(), fs_.as<double>(), f.data()));
        for (auto& q : rs) rc.push_back((q.a.nx * (long long)q.a.ny + kElemCells - 1) / kElemCells);
        res_.set(rs, rc);
    }
    std::vector<AsmSeg>    as;
    std::vector<long long> ac;
    std::vector<DstSeg>    di = dst_W_in_rec_, dout = dst_X_out_rec_;
    for (int g = 0; g < nd; ++g)
    {
        const Domain& D = dom_[g].d;
        AsmSeg        q{};
        q.f    = f[g];
        q.copy = ir ? fs_.as<double>() + dom_[g].off : nullptr;
        q.a.nx = D.nx;
        q.a.ny = D.ny;
        q.a.hx = D.hx;
        q.a.hy = D.hy;
        for (int k = 0; k < 4; ++k)
        {
            q.a.bc[k]    = D.bc[k];
            q.a.ghost[k] = gh.empty() ? nullptr : gh[4 * g + k];
        }
        as.push_back(q);
        ac.push_back((D.cells() + kAsmCells - 1) / kAsmCells);
        di[g].in   = f[g];
        dout[g].out = f[g];
    }
    asm_user_.set(as, ac);
    dst_user_in_.set(di, dst_kinds_, plans_);
    dst_user_out_.set(dout, dst_kinds_, plans_);
}

template <typename TS> ResSeg BatchImpl<TS>::res_seg(size_t g, double* r, const double* fs, const double* const* u_user)
{
    const Domain& D = dom_[g].d;
    ResSeg        q{};
    auto          U = [&](size_t h) -> const double* { return u_user[h]; };
    q.r    = r ? r + dom_[g].off : nullptr;
    q.fs   = fs + dom_[g].off;
    q.u    = U(g);
    q.a.nx = D.nx;
    q.a.ny = D.ny;
    q.a.r2 = D.hx * D.hx / D.hy / D.hy;
    for (int f = 0; f < 4; ++f)
    {
        q.a.bc[f] = D.bc[f];
        q.a.nb[f] = nullptr;
    }
    const Dom& d = dom_[g];
    const Prob& pr = prob_[d.prob];
    if (d.role == 1)
    {
        const Dom& R        = dom_[pr.root];
        q.a.nb[d.leaf_face] = U(pr.root);
        q.a.nbnx[d.leaf_face] = R.d.nx;
        q.a.nbny[d.leaf_face] = R.d.ny;
    }
    else
    {
        for (int h = pr.g0; h < pr.g0 + pr.nd; ++h)
        {
            if (dom_[h].role != 1) continue;
            const int f   = dom_[h].root_face;
            q.a.nb[f]     = U(h);
            q.a.nbnx[f]   = dom_[h].d.nx;
            q.a.nbny[f]   = dom_[h].d.ny;
        }
    }
    return q;
}

template <typename TS> void BatchImpl<TS>::run(int steps, cudaStream_t s)
{
    k_b_assemble<<<(unsigned)asm_user_.total, 256, 0, s>>>(asm_user_.as<AsmSeg>(), asm_user_.pre(), asm_user_.n);
    FPB_CHECK_LAUNCH();
    if (steps == 0)
    {
        inner(dst_user_in_, dst_user_out_, false, s);
        return;
    }
    first_inner(s);
    for (int k = 1; k < steps; ++k)
    {
        k_b_residual<<<(unsigned)res_.total, 256, 0, s>>>(res_.as<ResSeg>(), res_.pre(), res_.n);
        FPB_CHECK_LAUNCH();
        inner(dst_r_, dst_out_u_, true, s);
    }
}

template <typename TS>
void BatchImpl<TS>::solve(double* const* fields, const double* const* ghosts, int steps, cudaStream_t s)
{
    if (!fields) throw Error(1, "null field list");
    for (int g = 0; g < (int)dom_.size(); ++g)
        if (!fields[g]) throw Error(1, "null field pointer");
    if (steps < 0 || steps > 64) throw Error(1, "steps must be in [0, 64]");
    set_user_lists(fields, ghosts, steps);
    run(steps, s);
}

template <typename TS> void BatchImpl<TS>::solve_graph(double* const* fields, const double* const* ghosts, int steps,
                                                       cudaStream_t s)
{
    if (!fields) throw Error(1, "null field list");
    if (steps < 0 || steps > 64) throw Error(1, "steps must be in [0, 64]");
    set_user_lists(fields, ghosts, steps);
    if (!graph_)
    {
        cudaStream_t cap;
        FPB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g     = nullptr;
        const long long before = launches_noted();
        FPB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        try
        {
            run(steps, cap);
        }
        catch (...)
        {
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            throw;
        }
        FPB_CUDA(cudaStreamEndCapture(cap, &g));
        graph_kernels_ = launches_noted() - before;
        note_launches(-graph_kernels_);  // captured, not executed: counted when the graph is replayed
        const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        FPB_CUDA(e);
    }
    FPB_CUDA(cudaGraphLaunch(graph_, s));
    note_launches(graph_kernels_);
}

template <typename TS> void BatchImpl<TS>::prepare_assembled(const double* const* in, double* const* out)
{
    const int                  nd = (int)dom_.size();
    std::vector<const double*> vi(in, in + nd);
    std::vector<double*>       vo(out, out + nd);
    if (vi == ext_in_ && vo == ext_out_) return;
    FPB_CUDA(cudaDeviceSynchronize());  // the lists below may still be read by queued work
    std::vector<DstSeg> a = dst_W_in_rec_, b = dst_X_out_rec_;
    for (int g = 0; g < nd; ++g)
    {
        a[g].in  = vi[g];
        b[g].out = vo[g];
    }
    ext_in_list_.set(a, dst_kinds_, plans_);
    ext_out_list_.set(b, dst_kinds_, plans_);
    ext_in_  = vi;
    ext_out_ = vo;
    ++ext_gen_;
}

template <typename TS>
void BatchImpl<TS>::solve_assembled(const double* const* in, double* const* out, cudaStream_t s)
{
    prepare_assembled(in, out);
    inner(ext_in_list_, ext_out_list_, false, s);
}

// The refinement as one graph: assembly, the first solve (written straight into u), then a while node whose
// body is one correction (residual, inner solve, u += r with norms, k_ir_check, which ends the loop).
template <typename TS>
void BatchImpl<TS>::build_ir_graph(double rel_tol, int max_refine, BatchBase* first, const double* const* fi,
                                   double* const* fo)
{
    cudaStream_t cap = nullptr, cb = nullptr;
    cudaGraph_t  g   = nullptr;
    FPB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    const long long before = launches_noted();
    bool            in_cap = false, in_body = false;
    try
    {
        FPB_CUDA(cudaStreamCreateWithFlags(&cb, cudaStreamNonBlocking));
        FPB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        in_cap = true;
        k_b_assemble<<<(unsigned)asm_user_.total, 256, 0, cap>>>(asm_user_.as<AsmSeg>(), asm_user_.pre(), asm_user_.n);
        FPB_CHECK_LAUNCH();
        if (first) first->solve_assembled(fi, fo, cap);
        else first_inner(cap);
        k_ir_init<<<1, 1, 0, cap>>>(irst_.as<IrState>());
        FPB_CHECK_LAUNCH();
        ir_pro_ = launches_noted() - before;
        cudaStreamCaptureStatus  cs;
        cudaGraph_t              cg    = nullptr;
        const cudaGraphNode_t*   deps  = nullptr;
        size_t                   ndeps = 0;
        FPB_CUDA(cudaStreamGetCaptureInfo(cap, &cs, nullptr, &cg, &deps, &ndeps));
        cudaGraphConditionalHandle loop;
        FPB_CUDA(cudaGraphConditionalHandleCreate(&loop, cg, 1u, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np = {};
        np.type                = cudaGraphNodeTypeConditional;
        np.conditional.handle  = loop;
        np.conditional.type    = cudaGraphCondTypeWhile;
        np.conditional.size    = 1;
        cudaGraphNode_t node;
        FPB_CUDA(cudaGraphAddNode(&node, cg, deps, ndeps, &np));
        FPB_CUDA(cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies));
        FPB_CUDA(cudaStreamBeginCaptureToGraph(cb, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        in_body = true;
        k_b_residual<<<(unsigned)res_.total, 256, 0, cb>>>(res_.as<ResSeg>(), res_.pre(), res_.n);
        FPB_CHECK_LAUNCH();
        inner(dst_r_, dst_out_r_, false, cb);
        k_b_add_norms<<<(unsigned)addn_.total, 256, 0, cb>>>(addn_.as<AddSeg>(), addn_.pre(), addn_.n, 0);
        FPB_CHECK_LAUNCH();
        const long long nb = (long long)(addp_.bytes() / 16);
        k_ir_check<<<1, 256, 0, cb>>>(addp_.as<double>(), nb, irst_.as<IrState>(), rel_tol, max_refine, loop);
        FPB_CHECK_LAUNCH();
        cudaGraph_t body = nullptr;
        in_body          = false;
        FPB_CUDA(cudaStreamEndCapture(cb, &body));
        in_cap = false;
        FPB_CUDA(cudaStreamEndCapture(cap, &g));
        ir_body_ = launches_noted() - before - ir_pro_;
        note_launches(-(ir_pro_ + ir_body_));  // captured, not executed: counted per run from the steps taken
        const cudaError_t e = cudaGraphInstantiate(&irgraph_, g, 0);
        cudaGraphDestroy(g);
        g = nullptr;
        FPB_CUDA(e);
    }
    catch (...)
    {
        cudaGraph_t junk = nullptr;
        if (in_body) cudaStreamEndCapture(cb, &junk);
        if (in_cap) cudaStreamEndCapture(cap, &g);
        if (g) cudaGraphDestroy(g);
        note_launches(-(launches_noted() - before));
        irgraph_ = nullptr;
        if (cb) cudaStreamDestroy(cb);
        cudaStreamDestroy(cap);
        throw;
    }
    cudaStreamDestroy(cb);
    cudaStreamDestroy(cap);
    irfirst_ = first;
    irmax_   = max_refine;
    irtol_   = rel_tol;
    irgen_   = first ? first->assembled_generation() : 0;
}

// Reads the pinned copy of the refinement state after `runs` graph runs have completed: counts their
// kernels (the last run's steps for each) and reports a non-finite value met by any of them.
template <typename TS> int BatchImpl<TS>::ir_outcome(double* rel_change, long long runs)
{
    const IrState st = *irhost_;
    note_launches(runs * (ir_pro_ + ir_body_ * (long long)(st.steps - 1)));
    if (st.err_sticky)
    {
        FPB_CUDA(cudaMemset(&irst_.as<IrState>()->err_sticky, 0, sizeof(int)));
        irhost_->err_sticky = 0;
        throw Error(5, "non-finite value in iterative refinement");
    }
    last_steps_  = st.steps;
    last_change_ = st.change;
    if (rel_change) *rel_change = st.change;
    return st.steps;
}

template <typename TS> void BatchImpl<TS>::refine_result(int* steps, double* rel_change)
{
    if (!irhost_ || ir_pending_ == 0)
    {
        if (steps) *steps = last_steps_;
        if (rel_change) *rel_change = last_change_;
        return;
    }
    const long long runs = ir_pending_;
    ir_pending_          = 0;
    const int st         = ir_outcome(rel_change, runs);
    if (steps) *steps = st;
}

template <typename TS>
int BatchImpl<TS>::refine(double* const* fields, const double* const* ghosts, double rel_tol, int max_refine,
                         cudaStream_t s, double* rel_change, BatchBase* first, bool defer)
{
    if (!fields) throw Error(1, "null field list");
    if (!(rel_tol > 0) || max_refine < 1) throw Error(1, "rel_tol must be > 0 and max_refine >= 1");
    set_user_lists(fields, ghosts, 1);
    if (max_refine > 1)
    {
        const int                  nd = (int)dom_.size();
        std::vector<const double*> fi(nd);
        std::vector<double*>       fo(nd);
        for (int g = 0; g < nd; ++g)
        {
            fi[g] = fs_.as<double>() + dom_[g].off;
            fo[g] = user_ptrs_[g];
        }
        if (first) first->prepare_assembled(fi.data(), fo.data());
        if (!irst_.get())
        {
            irst_.alloc(sizeof(IrState));
            FPB_CUDA(cudaMemset(irst_.get(), 0, sizeof(IrState)));
            FPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&irhost_), sizeof(IrState)));
            *irhost_ = IrState{};
        }
        const long long gen = first ? first->assembled_generation() : 0;
        if (irgraph_ && (irfirst_ != first || irmax_ != max_refine || irtol_ != rel_tol || irgen_ != gen))
        {
            cudaGraphExecDestroy(irgraph_);
            irgraph_ = nullptr;
        }
        if (!irgraph_) build_ir_graph(rel_tol, max_refine, first, fi.data(), fo.data());
        FPB_CUDA(cudaGraphLaunch(irgraph_, s));
        FPB_CUDA(cudaMemcpyAsync(irhost_, irst_.get(), sizeof(IrState), cudaMemcpyDeviceToHost, s));
        if (defer)
        {
            ++ir_pending_;
            return -1;
        }
        FPB_CUDA(cudaStreamSynchronize(s));
        const long long runs = ir_pending_ + 1;
        ir_pending_          = 0;
        return ir_outcome(rel_change, runs);
    }
    // max_refine == 1: one inner solve into r, then u = r through the add pass, whose norms check the values
    k_b_assemble<<<(unsigned)asm_user_.total, 256, 0, s>>>(asm_user_.as<AsmSeg>(), asm_user_.pre(), asm_user_.n);
    FPB_CHECK_LAUNCH();
    if (first)
    {
        std::vector<const double*> fi(dom_.size());
        std::vector<double*>       ro(dom_.size());
        for (size_t g = 0; g < dom_.size(); ++g)
        {
            fi[g] = fs_.as<double>() + dom_[g].off;
            ro[g] = r_.as<double>() + dom_[g].off;
        }
        first->solve_assembled(fi.data(), ro.data(), s);
    }
    else
        inner(dst_fs_, dst_out_r_, false, s);
    k_b_add_norms<<<(unsigned)addn_.total, 256, 0, s>>>(addn_.as<AddSeg>(), addn_.pre(), addn_.n, 1);
    FPB_CHECK_LAUNCH();
    const long long     nb = (long long)(addp_.bytes() / 16);
    std::vector<double> hp((size_t)2 * nb);
    FPB_CUDA(cudaMemcpyAsync(hp.data(), addp_.get(), hp.size() * 8, cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
    double cn = 0, un = 0;
    for (long long b = 0; b < nb; ++b)
    {
        cn += hp[b];
        un += hp[nb + b];
    }
    if (!std::isfinite(cn) || !std::isfinite(un)) throw Error(5, "non-finite value in iterative refinement");
    last_steps_  = 1;
    last_change_ = un > 0 ? std::sqrt(cn / un) : 0.0;
    if (rel_change) *rel_change = last_change_;
    return 1;
}

template <typename TS>
void BatchImpl<TS>::residuals(const double* const* u, const double* const* rhs, const double* const* ghosts,
                              cudaStream_t s, double* out)
{
    const int nd = (int)dom_.size();
    DevBuf    fs((size_t)cells_ * 8);
    std::vector<AsmSeg>    as;
    std::vector<ResSeg>    rs;
    std::vector<long long> ac, bo(nd + 1, 0);
    for (int g = 0; g < nd; ++g)
    {
        const Domain& D = dom_[g].d;
        AsmSeg        q{};
        q.f    = const_cast<double*>(rhs[g]);
        q.copy = fs.as<double>() + dom_[g].off;
        q.a.nx = D.nx;
        q.a.ny = D.ny;
        q.a.hx = D.hx;
        q.a.hy = D.hy;
        for (int k = 0; k < 4; ++k)
        {
            q.a.bc[k]    = D.bc[k];
            q.a.ghost[k] = ghosts ? ghosts[4 * g + k] : nullptr;
        }
        as.push_back(q);
        ac.push_back((D.cells() + kElemCells - 1) / kElemCells);
        bo[g + 1] = bo[g] + ac.back();
    }
    std::vector<long long> acb;
    for (int g = 0; g < nd; ++g) acb.push_back((dom_[g].d.cells() + kAsmCells - 1) / kAsmCells);
    DevBuf pa((size_t)bo[nd] * 8), pf((size_t)bo[nd] * 8);
    for (int g = 0; g < nd; ++g)
    {
        ResSeg q      = res_seg(g, nullptr, fs.as<double>(), u);
        q.fs          = fs.as<double>() + dom_[g].off;
        q.partial     = pa.as<double>() + bo[g];
        q.partial_f   = pf.as<double>() + bo[g];
        rs.push_back(q);
    }
    Segments A, R;
    A.set(as, acb);
    R.set(rs, ac);
    k_b_assemble<<<(unsigned)A.total, 256, 0, s>>>(A.as<AsmSeg>(), A.pre(), A.n);
    FPB_CHECK_LAUNCH();
    k_b_residual<<<(unsigned)R.total, 256, 0, s>>>(R.as<ResSeg>(), R.pre(), R.n);
    FPB_CHECK_LAUNCH();
    std::vector<double> ha(bo[nd]), hf(bo[nd]);
    FPB_CUDA(cudaMemcpyAsync(ha.data(), pa.get(), ha.size() * 8, cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaMemcpyAsync(hf.data(), pf.get(), hf.size() * 8, cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
    for (size_t p = 0; p < prob_.size(); ++p)
    {
        double rr = 0, ff = 0;
        for (int g = prob_[p].g0; g < prob_[p].g0 + prob_[p].nd; ++g)
            for (long long b = bo[g]; b < bo[g + 1]; ++b)
            {
                rr += ha[b];
                ff += hf[b];
            }
        out[p] = ff > 0 ? std::sqrt(rr / ff) : std::sqrt(rr);
    }
}

// Launch shapes by measurement: the DST over all subdomains (threads per CTA x CTAs per SM) and the
// chase (threads per CTA), each candidate timed with CUDA events on the real work lists (contents of
// the work buffers are irrelevant to the timing; they are zeroed first).
template <typename TS> void BatchImpl<TS>::autotune(cudaStream_t s)
{
    FPB_CUDA(cudaMemsetAsync(W_.get(), 0, (size_t)cells_ * sizeof(TS), s));
    FPB_CUDA(cudaMemsetAsync(X_.get(), 0, (size_t)cells_ * sizeof(TS), s));
    std::vector<DstSeg> rec = dst_X_out_rec_;
    for (size_t g = 0; g < dom_.size(); ++g) rec[g].out = W_.as<TS>() + dom_[g].off;
    XList sg;
    sg.set(rec, dst_kinds_, plans_);
    cudaEvent_t e0, e1;
    FPB_CUDA(cudaEventCreate(&e0));
    FPB_CUDA(cudaEventCreate(&e1));
    auto time_it = [&](auto&& fn) {
        fn();
        FPB_CUDA(cudaEventRecord(e0, s));
        for (int r = 0; r < 3; ++r) fn();
        FPB_CUDA(cudaEventRecord(e1, s));
        FPB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        FPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    };
    BatchTiming best = tm_;
    float       bt   = 1e30f;
    for (int th : {128, 192, 256, 384, 512})
    {
        int occ = 0;
        FPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_xform<TS, K_DD, 0, TS, TS, false, 0>, th,
                                                               plans_.smem));
        // persistent grids of 1, 2, 4, the occupancy limit CTAs per SM, or one CTA per work item (1 << 20)
        for (int bps : {1, 2, 4, occ, 1 << 20})
        {
            if (bps < 1 || (bps > occ && bps != (1 << 20))) continue;
            tm_.dst_threads       = th;
            tm_.dst_blocks_per_sm = bps;
            const float t = time_it([&] { launch_x<TS, TS, TS, false>(sg, false, plans_, tm_, s); });
            if (t < bt)
            {
                bt   = t;
                best = tm_;
            }
        }
    }
    tm_ = best;
    bt  = 1e30f;
    for (int th : {128, 256})
    {
        tm_.chase_threads = th;
        build_chase_lists();
        const float t = time_it([&] { chase_run(a2_lc_, a2_red_, s); });
        if (t < bt)
        {
            bt                 = t;
            best.chase_threads = th;
        }
    }
    tm_ = best;
    build_chase_lists();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs();
}

// Captured graphs hold the work lists and launch shapes of their capture; an executable graph still in flight
// is released when it completes.
template <typename TS> void BatchImpl<TS>::drop_graphs()
{
    if (graph_) cudaGraphExecDestroy(graph_);
    if (irgraph_) cudaGraphExecDestroy(irgraph_);
    graph_   = nullptr;
    irgraph_ = nullptr;
}

std::unique_ptr<BatchBase> make_batch(const std::vector<BatchProblemDesc>& probs, int precision)
{
    if (precision == 1) return std::unique_ptr<BatchBase>(new BatchImpl<float>(probs));
    return std::unique_ptr<BatchBase>(new BatchImpl<double>(probs));
}

}  // namespace fpb
