// Small device operations of the composite solve: boundary assembly and h^2 scaling, interface
// coupling (bond_add), edge gather/scatter, dense Schur matrix-vector products, deterministic BLAS-1.
// Included by more than one translation unit: the non-template kernels have internal linkage.
#pragma once

#include "fp_common.cuh"

namespace fpb
{

// Edge element k of face `loc` of an nx x ny field: XNEG row 0, XPOS row nx-1, YNEG column 0,
// YPOS column ny-1 (field2::*_bond_add, base/field/field2.cpp:212-302).
__host__ __device__ __forceinline__ long long edge_index(int loc, int nx, int ny, int k)
{
    switch (loc)
    {
        case 0: return k;
        case 1: return (long long)(nx - 1) * ny + k;
        case 2: return (long long)k * ny;
        default: return (long long)k * ny + (ny - 1);
    }
}
__host__ __device__ __forceinline__ int edge_length(int loc, int nx, int ny) { return loc < 2 ? ny : nx; }

struct AssembleArgs
{
    int           nx, ny;
    double        hx, hy;
    int           bc[4];
    const double* ghost[4];  // may be null (zero ghost values)
};

// f = (f + boundary terms) * hx^2 in the order of ConcatPoissonSolver2D::boundary_assembly
// (pe/concat/concat_solver2d.cpp:159-223: Dirichlet faces x-,x+,y-,y+ then Neumann faces) followed by
// the hx^2 scaling of solve() (:111-116).
template <typename T> __device__ __forceinline__ void assemble_at(T* __restrict__ f, long long t, const AssembleArgs& a)
{
    const int i = (int)t / a.ny, j = (int)t - i * a.ny;  // a subdomain holds fewer than 2^31 cells
    double    v = f[t];
    const bool on[4] = {i == 0, i == a.nx - 1, j == 0, j == a.ny - 1};
    if (on[0] || on[1] || on[2] || on[3])
    {
        const int    idx[4] = {j, j, i, i};
        const double dco[4] = {-1.0 / a.hx / a.hx, -1.0 / a.hx / a.hx, -1.0 / a.hy / a.hy, -1.0 / a.hy / a.hy};
        const double nco[4] = {1.0 / a.hx, -1.0 / a.hx, 1.0 / a.hy, -1.0 / a.hy};
        for (int face = 0; face < 4; ++face)
            if (on[face] && a.bc[face] == 0) v += dco[face] * (a.ghost[face] ? a.ghost[face][idx[face]] : 0.0);
        for (int face = 0; face < 4; ++face)
            if (on[face] && a.bc[face] == 1) v += nco[face] * (a.ghost[face] ? a.ghost[face][idx[face]] : 0.0);
    }
    f[t] = (T)(v * (a.hx * a.hx));
}
template <typename T> __global__ void k_assemble_scale(T* __restrict__ f, const AssembleArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nx * a.ny) return;
    assemble_at(f, t, a);
}

// dst.bond_add(loc, a, src): dst's face `loc` += a * src's opposite face (field2.cpp:257-302).
template <typename T>
__global__ void k_bond_add(T* __restrict__ dst, int dnx, int dny, int loc, T a, const T* __restrict__ src, int snx,
                           int sny)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = edge_length(loc, dnx, dny);
    if (k >= n) return;
    const long long di = edge_index(loc, dnx, dny, k);
    const long long si = edge_index(loc ^ 1, snx, sny, k);
    dst[di] += a * src[si];
}

// out[k] = v[k] - field.edge(loc)[k]   (GMRES Afun: x - ft restricted to the interface)
template <typename T>
__global__ void k_edge_sub(T* __restrict__ out, const T* __restrict__ v, const T* __restrict__ field, int nx, int ny,
                           int loc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = edge_length(loc, nx, ny);
    if (k >= n) return;
    out[k] = v[k] + (T)-1.0 * field[edge_index(loc, nx, ny, k)];
}

// out[k] = field.edge(loc)[k]
template <typename T>
__global__ void k_edge_gather(T* __restrict__ out, const T* __restrict__ field, int nx, int ny, int loc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = edge_length(loc, nx, ny);
    if (k >= n) return;
    out[k] = field[edge_index(loc, nx, ny, k)];
}

// field.edge(loc)[i] += sum_j S[i*cn + j] * v[j * vstride]  -- one warp per row i
// (SchurMat2D_*::operator*, pe/concat/schur_mat2d.cpp:18-123). v may be a field edge (vstride = the
// edge's element stride) or a contiguous interface vector (vstride = 1).
template <typename T>
__global__ void k_schur_matvec(const double* __restrict__ S, int cn, const T* __restrict__ v, long long vstride,
                               T* __restrict__ field, int nx, int ny, int loc)
{
    const int row  = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= cn) return;
    const double* Sr  = S + (long long)row * cn;
    double        acc = 0.0;
    for (int j = lane; j < cn; j += 32) acc += (double)v[j * vstride] * Sr[j];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0)
    {
        const long long e = edge_index(loc, nx, ny, row);
        field[e]          = (T)((double)field[e] + acc);
    }
}

// Impulse batch for Schur construction: fields[b] (zeroed by the caller) gets 1 at interface cell
// i0 + b of face `loc` (SchurMat2D_*::construct, schur_mat2d.cpp:5-16).
template <typename T> __global__ void k_impulses(T* fields, int nx, int ny, int loc, int i0, int nb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    fields[(long long)b * nx * ny + edge_index(loc, nx, ny, i0 + b)] = (T)1;
}
// S[j*cn + (i0+b)] = fields[b].edge(loc)[j]
template <typename T>
__global__ void k_impulse_extract(const T* fields, int nx, int ny, int loc, double* S, int cn, int i0, int nb)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * cn) return;
    const int b = (int)(t / cn), j = (int)(t % cn);
    S[(long long)j * cn + i0 + b] = (double)fields[(long long)b * nx * ny + edge_index(loc, nx, ny, j)];
}

// ---------------------------------------------------------------------------------------------
// Deterministic BLAS-1 on FP64 vectors. Reductions: fixed grid, per-block partial sums, the last
// block (atomic ticket, no waiting) adds the partials in index order.
// ---------------------------------------------------------------------------------------------
constexpr int kRedBlocks  = 256;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    return s;
}

// out[0] = sum_i a[i] * b[i]  (b == a: squared norm). partials: kRedBlocks doubles; ticket: 1 uint (zero)
static __global__ void k_dot(const double* __restrict__ a, const double* __restrict__ b, long long n, double* partials,
                      unsigned* ticket, double* out, int take_sqrt)
{
    __shared__ double sh[32];
    __shared__ bool   last;
    double            v = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v += a[i] * b[i];
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        double tot = 0;
        for (int k = 0; k < (int)gridDim.x; ++k) tot += ((volatile double*)partials)[k];
        *out    = take_sqrt ? sqrt(tot) : tot;
        *ticket = 0u;
    }
}

// y += coef * x, coef = sign * (*c)  (coefficient read from device memory)
static __global__ void k_axpy_dev(double* __restrict__ y, const double* __restrict__ x, long long n, const double* c, double sign)
{
    const double a = sign * (*c);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}
// y = (1 / *h) * x + 0
static __global__ void k_scale_inv(double* __restrict__ y, const double* __restrict__ x, long long n, const double* h)
{
    const double a = 1.0 / (*h);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = 0.0 + a * x[i];
}
// r = b + (-1) * ax
static __global__ void k_sub(double* __restrict__ r, const double* __restrict__ b, const double* __restrict__ ax, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r[i] = b[i] + -1.0 * ax[i];
}
// x += y_0 V_0 + y_1 V_1 + ... (applied in order per element, like sequential axpys)
static __global__ void k_multi_axpy(double* __restrict__ x, const double* __restrict__ V, long long ld, long long n,
                             const double* __restrict__ y, int k)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        double v = x[i];
        for (int q = 0; q < k; ++q) v += y[q] * V[q * ld + i];
        x[i] = v;
    }
}
// y *= a
static __global__ void k_scale(double* __restrict__ y, double a, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] *= a;
}
// y += x (mixed precision: T field added into a double field)
template <typename T>
__global__ void k_add(double* __restrict__ y, const T* __restrict__ x, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += (double)x[i];
}

}  // namespace fpb

namespace fpb
{
// ---------------------------------------------------------------------------------------------
// Dense interface operator and its inverse (preconditioner of the interface GMRES)
// ---------------------------------------------------------------------------------------------
// fields[b].edge(loc)[q] = S[q*cn + c0 + b]: column c0+b of a child's Schur matrix placed on the edge
static __global__ void k_edge_scatter_col(double* fields, long long cells, int nx, int ny, int loc, const double* S, int cn,
                                   int c0, int nb)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * cn) return;
    const int b = (int)(t / cn), q = (int)(t % cn);
    fields[b * cells + edge_index(loc, nx, ny, q)] = S[(long long)q * cn + c0 + b];
}
// K[(off+q)*ld + c0 + b] = fields[b].edge(loc)[q]
static __global__ void k_edge_gather_col(double* K, long long ld, int off, const double* fields, long long cells, int nx,
                                  int ny, int loc, int cn, int c0, int nb)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * cn) return;
    const int b = (int)(t / cn), q = (int)(t % cn);
    K[(long long)(off + q) * ld + c0 + b] = fields[b * cells + edge_index(loc, nx, ny, q)];
}
// A = I - A (n x n)
static __global__ void k_identity_minus(double* A, int n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const long long i = t / n, j = t % n;
    A[t]              = (i == j ? 1.0 : 0.0) - A[t];
}
// A = 2I - A (n x n)
static __global__ void k_two_identity_minus(double* A, int n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const long long i = t / n, j = t % n;
    A[t]              = (i == j ? 2.0 : 0.0) - A[t];
}
// X = s * M^T (row-major n x n)
static __global__ void k_scaled_transpose(double* X, const double* M, int n, double s)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const long long i = t / n, j = t % n;
    X[t]              = s * M[j * n + i];
}
// rowsum[i] = sum_j |A[i][j]| and colsum[j] = sum_i |A[i][j]| (one thread per row / column)
static __global__ void k_abs_sums(const double* A, int n, double* rowsum, double* colsum)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double r = 0, c = 0;
    for (int k = 0; k < n; ++k)
    {
        r += fabs(A[(long long)t * n + k]);
        c += fabs(A[(long long)k * n + t]);
    }
    rowsum[t] = r;
    colsum[t] = c;
}
// out[0] = sum_{ij} (I - P)_{ij}^2 (deterministic: per-block partials, last block adds them in order)
static __global__ void k_identity_residual(const double* __restrict__ P, int n, double* partials, unsigned* ticket,
                                    double* out)
{
    __shared__ double sh[32];
    __shared__ bool   last;
    double            v     = 0;
    const long long   total = (long long)n * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x)
    {
        const double e = ((t / n) == (t % n) ? 1.0 : 0.0) - P[t];
        v += e * e;
    }
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        double tot = 0;
        for (int k = 0; k < (int)gridDim.x; ++k) tot += ((volatile double*)partials)[k];
        *out    = tot;
        *ticket = 0u;
    }
}
// y (+)= X g, row-major n x n, one warp per row
static __global__ void k_dense_matvec(const double* __restrict__ X, int n, const double* __restrict__ g,
                               double* __restrict__ y, int accumulate)
{
    const int row  = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double* Xr  = X + (long long)row * n;
    double        acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += Xr[j] * g[j];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) y[row] = accumulate ? y[row] + acc : acc;
}
// r = g - y + field.edge(loc)   on one child's interface block
static __global__ void k_interface_residual(double* r, const double* g, const double* y, const double* field, int nx, int ny,
                                     int loc, int cn)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cn) return;
    r[k] = g[k] - y[k] + field[edge_index(loc, nx, ny, k)];
}
}  // namespace fpb

namespace fpb
{
// ---------------------------------------------------------------------------------------------
// FP64 residual of the composite 5-point operator (iterative refinement)
// ---------------------------------------------------------------------------------------------
struct ResidualArgs
{
    int           nx, ny;
    double        r2;         // (hx/hy)^2
    int           bc[4];      // with Adjacented on connected faces
    const double* nb[4];      // neighbour fields on Adjacented faces
    int           nbnx[4], nbny[4];
};

// r = fs - A u with (A u)_ij = u_{i-1,j} + u_{i+1,j} - 2u_ij + r2 (u_{i,j-1} + u_{i,j+1} - 2u_ij): ghosts 0
// (Dirichlet), mirrored (Neumann), wrapped (periodic); an Adjacented face contributes the neighbour's
// adjacent cell with coefficient 1 -- the operator ConcatPoissonSolver2D::solve inverts
// (pe/concat/concat_solver2d.cpp:101-157, interface terms from bond_add with coefficient -1).
//
// The residual is computed in double-FP64 ("double-double") arithmetic and rounded once. For a smooth
// solution the stencil's terms are ~cond(A) times larger than their sum, and a plain FP64 sum carries an
// error of eps * |terms|: the computed residual of the exact solution would then be ~eps * cond(A)
// relative (1e-8 at h = 1/4096), and iterative refinement on it cannot get below that. Here every sum is
// exact to second order (TwoSum; products by r2 through an FMA remainder), so the residual is accurate to
// ~eps relative to itself and refinement converges to the solution's own FP64 rounding.
// The _rn intrinsics are never contracted into FMAs, which would break the error-free transformations.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e)
{
    s              = __dadd_rn(a, b);
    const double v = __dsub_rn(s, a);
    e              = __dadd_rn(__dsub_rn(a, __dsub_rn(s, v)), __dsub_rn(b, v));
}
__device__ __forceinline__ void dd_acc(double& hi, double& lo, double x)
{
    double s, e;
    two_sum(hi, x, s, e);
    hi = s;
    lo += e;
}
__device__ __forceinline__ void dd_acc_prod(double& hi, double& lo, double a, double b)
{
    const double p = __dmul_rn(a, b);
    dd_acc(hi, lo, p);
    lo += fma(a, b, -p);
}

// fs_t - (A u)_t, compensated as above.
__device__ __forceinline__ double composite_residual_at(const double* __restrict__ u, double fs, long long t,
                                                        const ResidualArgs& a)
{
    const int    i = (int)t / a.ny, j = (int)t - i * a.ny;  // a subdomain holds fewer than 2^31 cells
    const int    nx = a.nx, ny = a.ny;
    const double c  = u[t];
    double       wym = a.r2, wyp = a.r2;  // y neighbours' weights: 1 across an Adjacented face
    auto ghost = [&](int face, int k, double own, double wrap, double& w) -> double {
        switch (a.bc[face])
        {
            case 0: return 0.0;
            case 1: return own;
            case 2: return wrap;
            default:
            {
                w = 1.0;
                return a.nb[face][edge_index(face ^ 1, a.nbnx[face], a.nbny[face], k)];
            }
        }
    };
    double       wx = 1.0;
    const double xm = (i > 0) ? u[t - ny] : ghost(0, j, c, u[(long long)(nx - 1) * ny + j], wx);
    const double xp = (i < nx - 1) ? u[t + ny] : ghost(1, j, c, u[j], wx);
    const double ym = (j > 0) ? u[t - 1] : ghost(2, i, c, u[(long long)i * ny + ny - 1], wym);
    const double yp = (j < ny - 1) ? u[t + 1] : ghost(3, i, c, u[(long long)i * ny], wyp);
    double       hi = xm, lo = 0.0;
    dd_acc(hi, lo, xp);
    dd_acc(hi, lo, -2.0 * c);
    dd_acc_prod(hi, lo, wym, ym);
    dd_acc_prod(hi, lo, wyp, yp);
    dd_acc_prod(hi, lo, a.r2, -2.0 * c);
    double s, e;
    two_sum(fs, -hi, s, e);
    return s + (e - lo);
}
static __global__ void k_composite_residual(double* __restrict__ r, const double* __restrict__ fs,
                                            const double* __restrict__ u, const ResidualArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nx * a.ny) return;
    r[t] = composite_residual_at(u, fs[t], t, a);
}
}  // namespace fpb
