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

template <typename T>
__global__ void k_chase(T* __restrict__ f, int nx, int ny, long long batch, const T* __restrict__ ctab,
                        const T* __restrict__ z1, const T* __restrict__ z2, int periodic, int singular)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= batch * ny) return;
    const int       j   = (int)(t % ny);
    const long long b   = t / ny;
    T*              col = f + b * (long long)nx * ny + j;
    const long long s   = ny;

    if (singular && j == ny - 1)
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
