// GMRES(m) control on the device: the restart loop of the reference's GMRESSolver2D / GMRESSolver3D
// (pe/concat/gmres_solver2d.cpp:120-252, gmres_solver3d.cpp:155-306) as one CUDA graph with three nested
// conditional WHILE nodes (restarts, Arnoldi steps, modified Gram-Schmidt projections) whose conditions these
// kernels set. Every loop is bounded by construction: the restart loop by max_iter, the Arnoldi loop by m, the
// projection loop by the step index; a non-finite value clears the conditions and sets err. The arithmetic is
// the host loop's (same reductions, same Givens and back-substitution order), so the iterates are the same.
#pragma once

#include "fp_internal.h"
#include "fp_ops.cuh"

#include <cuda_runtime.h>

namespace fpb
{
struct GmState
{
    int    outer, j, i, active, converged, err, iters, restarts;
    double beta, inner_tol;
};
struct GmArrays  // (m + 1) x m Hessenberg, rotations, right-hand side, solution, current column
{
    double *H, *cs, *sn, *g, *y, *hcol;
};

namespace
{

__global__ void k_gm_start(GmState* st)
{
    st->outer     = 0;
    st->converged = 0;
    st->err       = 0;
    st->iters     = 0;
    st->restarts  = 0;
    st->active    = 0;
}

// After the residual norms: the restart test and the new Krylov start. hcol[m + 1] = ||r|| of the Krylov
// vectors; with `interface` the test is on the full-field residual norm in hcol[m] and the inner test on
// |g_{j+1}| is scaled by their ratio (the 2D interface mode), else both use ||r|| (gmres_solver2d.cpp:149-160,
// gmres_solver3d.cpp:183-196).
__global__ void k_gm_check(GmState* st, GmArrays a, int m, double tol, int interface, cudaGraphConditionalHandle inner)
{
    const double rho  = a.hcol[m + 1];
    const double beta = interface ? a.hcol[m] : rho;
    st->beta          = beta;
    st->j             = 0;
    if (!isfinite(beta) || !isfinite(rho))
    {
        st->err    = 1;
        st->active = 0;
    }
    else if (beta < tol)
    {
        st->converged = 1;
        st->active    = 0;
    }
    else
    {
        st->active    = 1;
        st->inner_tol = (interface && beta > 0) ? 0.5 * tol * (rho / beta) : tol;
        st->restarts += 1;
        for (int q = 0; q < (m + 1) * m; ++q) a.H[q] = 0.0;
        for (int q = 0; q < m; ++q) a.cs[q] = a.sn[q] = 0.0;
        for (int q = 0; q <= m; ++q) a.g[q] = 0.0;
        a.g[0] = rho;
    }
    cudaGraphSetConditional(inner, st->active ? 1u : 0u);
}

// V0 = r * (1 / ||r||) when the restart goes on
__global__ void k_gm_start_basis(double* __restrict__ V, const double* __restrict__ r, long long n, const GmState* st,
                                 const double* hres)
{
    if (!st->active) return;
    const double a = 1.0 / (*hres);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        V[i] = r[i] * a;
}

// vin = V_j (the Arnoldi step's input in a fixed buffer); then the projection loop starts at i = 0
__global__ void k_gm_take(double* __restrict__ vin, const double* __restrict__ V, long long n, GmState* st)
{
    const double* v = V + (long long)st->j * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        vin[i] = v[i];
}
__global__ void k_gm_mgs_begin(GmState* st, cudaGraphConditionalHandle mgs)
{
    st->i = 0;
    cudaGraphSetConditional(mgs, 1u);
}

// hcol[idx] = a . b with a = V_{st->i} (which = 0) or w (which = 1, idx = j + 1, take the square root)
__global__ void k_gm_dot(const double* __restrict__ V, const double* __restrict__ w, long long n, const GmState* st,
                         double* hcol, double* partials, unsigned* ticket, int which)
{
    __shared__ double sh[32];
    __shared__ bool   last;
    const double*     a = which ? w : V + (long long)st->i * n;
    double            v = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v += a[i] * w[i];
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
        if (which) hcol[st->j + 1] = sqrt(tot);
        else hcol[st->i] = tot;
        *ticket = 0u;
    }
}
// w -= hcol[i] V_i, then i += 1 and the projection loop goes on while i <= j
__global__ void k_gm_axpy(double* __restrict__ w, const double* __restrict__ V, long long n, const GmState* st,
                          const double* hcol)
{
    const double  c = -hcol[st->i];
    const double* v = V + (long long)st->i * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        w[i] += c * v[i];
}
__global__ void k_gm_mgs_next(GmState* st, cudaGraphConditionalHandle mgs)
{
    st->i += 1;
    cudaGraphSetConditional(mgs, st->i <= st->j ? 1u : 0u);
}

// V_{j+1} = w / ||w|| (unused after a breakdown)
__global__ void k_gm_next_basis(double* __restrict__ V, const double* __restrict__ w, long long n, const GmState* st,
                                const double* hcol)
{
    const double a = 1.0 / hcol[st->j + 1];
    double*      v = V + (long long)(st->j + 1) * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = 0.0 + a * w[i];
}

// The Arnoldi step's scalar part (gmres_solver2d.cpp:188-225, gmres_solver3d.cpp:233-268): H column, breakdown
// test, Givens rotations, the inner test on |g_{j+1}|
__global__ void k_gm_arnoldi(GmState* st, GmArrays a, int m, cudaGraphConditionalHandle inner)
{
    const int    j = st->j;
    const double h = a.hcol[j + 1];
    if (!isfinite(h))
    {
        st->err    = 1;
        st->active = 0;
        cudaGraphSetConditional(inner, 0u);
        return;
    }
    st->iters += 1;
    for (int i = 0; i <= j; ++i) a.H[i * m + j] = a.hcol[i];
    if (h < 1e-12)
    {
        cudaGraphSetConditional(inner, 0u);  // breakdown: j columns
        return;
    }
    a.H[(j + 1) * m + j] = h;
    for (int i = 0; i < j; ++i)
    {
        const double t       = a.cs[i] * a.H[i * m + j] + a.sn[i] * a.H[(i + 1) * m + j];
        a.H[(i + 1) * m + j] = -a.sn[i] * a.H[i * m + j] + a.cs[i] * a.H[(i + 1) * m + j];
        a.H[i * m + j]       = t;
    }
    const double hjj = a.H[j * m + j], hj1 = a.H[(j + 1) * m + j];
    const double den = hypot(hjj, hj1);
    a.cs[j]          = hjj / den;
    a.sn[j]          = hj1 / den;
    a.H[j * m + j]       = a.cs[j] * a.H[j * m + j] + a.sn[j] * a.H[(j + 1) * m + j];
    a.H[(j + 1) * m + j] = 0.0;
    const double t       = a.cs[j] * a.g[j];
    a.g[j + 1]           = -a.sn[j] * a.g[j];
    a.g[j]               = t;
    st->j                = j + 1;
    cudaGraphSetConditional(inner, (fabs(a.g[j + 1]) < st->inner_tol || j + 1 >= m) ? 0u : 1u);
}

// y by back substitution (gmres_solver3d.cpp:281-290)
__global__ void k_gm_solve_y(GmState* st, GmArrays a, int m)
{
    if (!st->active) return;
    const int j = st->j;
    for (int i = 0; i < m; ++i) a.y[i] = 0.0;
    for (int i = j - 1; i >= 0; --i)
    {
        double v = a.g[i];
        for (int k = i + 1; k < j; ++k) v -= a.H[i * m + k] * a.y[k];
        a.y[i] = v / a.H[i * m + i];
    }
}
// x += y_0 V_0 + ... + y_{j-1} V_{j-1}, in the reference's order per element
__global__ void k_gm_update(double* __restrict__ x, const double* __restrict__ V, long long n, const GmState* st,
                            const double* __restrict__ y)
{
    if (!st->active) return;
    const int k = st->j;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        double v = x[i];
        for (int q = 0; q < k; ++q) v += y[q] * V[q * n + i];
        x[i] = v;
    }
}
// the restart loop goes on while not converged and outer < max_iter
__global__ void k_gm_outer_next(GmState* st, int max_iter, cudaGraphConditionalHandle outer)
{
    st->outer += 1;
    cudaGraphSetConditional(outer, (st->active && !st->err && st->outer < max_iter) ? 1u : 0u);
}


struct GmBuffers  // device buffers of one GMRES: Krylov basis V ((m + 1) x n), w, r, x, b, the step's input vin
{
    double *  V, *w, *r, *x, *b, *vin;
    GmState*  st;
    GmArrays  a;
    double*   partials;  // reduction scratch of dot(): kRedBlocks doubles and a ticket
    unsigned* ticket;
};

// Conditional WHILE node after the work captured so far on `cap`, controlled by `h`; its body is then captured
// on `body`.
inline void gm_while(cudaStream_t cap, cudaStream_t body, cudaGraphConditionalHandle h)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t             cg    = nullptr;
    const cudaGraphNode_t*  deps  = nullptr;
    size_t                  ndeps = 0;
    FPB_CUDA(cudaStreamGetCaptureInfo(cap, &cs, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams np = {};
    np.type                = cudaGraphNodeTypeConditional;
    np.conditional.handle  = h;
    np.conditional.type    = cudaGraphCondTypeWhile;
    np.conditional.size    = 1;
    cudaGraphNode_t node;
    FPB_CUDA(cudaGraphAddNode(&node, cg, deps, ndeps, &np));
    FPB_CUDA(cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies));
    FPB_CUDA(cudaStreamBeginCaptureToGraph(body, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
}
// A conditional handle on the graph being captured on `cap`.
inline cudaGraphConditionalHandle gm_handle(cudaStream_t cap, unsigned dflt, bool assign)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t             cg = nullptr;
    FPB_CUDA(cudaStreamGetCaptureInfo(cap, &cs, nullptr, &cg, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    FPB_CUDA(cudaGraphConditionalHandleCreate(&h, cg, dflt, assign ? cudaGraphCondAssignDefault : 0));
    return h;
}

// Captures and instantiates the GMRES(m) loop for (I - A^-1 S) x = A^-1 b on vectors of length n: afun(in, out, q)
// queues out = that operator applied to in; extra(q) queues, in interface mode, the full-field residual norm
// into a.hcol[m] (after r is formed); dot(x, y, len, sqrt, out, q) queues a reduction into a device scalar. The
// graph reads b and x from B on every launch and leaves the solution in x and the outcome in *B.st. The
// work afun and extra capture must allocate nothing (callers run them once beforehand).
template <typename Afun, typename Extra, typename Dot>
cudaGraphExec_t capture_gmres(long long n, int m, double tol, int max_iter, bool interface, const GmBuffers& B,
                              Afun afun, Extra extra, Dot dot)
{
    cudaStream_t q[4] = {};
    for (auto& x : q) FPB_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    const long long before = launches_noted();
    auto            grid   = [](long long len, int block, int cap) {
        const long long g = (len + block - 1) / block;
        return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
    };
    cudaGraph_t     g     = nullptr;
    int             depth = 0;
    cudaGraphExec_t exec  = nullptr;
    try
    {
        FPB_CUDA(cudaStreamBeginCapture(q[0], cudaStreamCaptureModeThreadLocal));
        depth = 1;
        k_gm_start<<<1, 1, 0, q[0]>>>(B.st);
        FPB_CHECK_LAUNCH();
        const cudaGraphConditionalHandle outer = gm_handle(q[0], 1u, true);
        gm_while(q[0], q[1], outer);
        depth = 2;
        afun(B.x, B.w, q[1]);
        k_sub<<<grid(n, 256, 4096), 256, 0, q[1]>>>(B.r, B.b, B.w, n);
        FPB_CHECK_LAUNCH();
        dot(B.r, B.r, n, true, B.a.hcol + m + 1, q[1]);
        extra(q[1]);
        const cudaGraphConditionalHandle inner = gm_handle(q[1], 0u, false);
        k_gm_check<<<1, 1, 0, q[1]>>>(B.st, B.a, m, tol, interface ? 1 : 0, inner);
        FPB_CHECK_LAUNCH();
        k_gm_start_basis<<<grid(n, 256, 4096), 256, 0, q[1]>>>(B.V, B.r, n, B.st, B.a.hcol + m + 1);
        FPB_CHECK_LAUNCH();
        gm_while(q[1], q[2], inner);
        depth = 3;
        k_gm_take<<<grid(n, 256, 4096), 256, 0, q[2]>>>(B.vin, B.V, n, B.st);
        FPB_CHECK_LAUNCH();
        afun(B.vin, B.w, q[2]);
        const cudaGraphConditionalHandle mgs = gm_handle(q[2], 0u, false);
        k_gm_mgs_begin<<<1, 1, 0, q[2]>>>(B.st, mgs);
        FPB_CHECK_LAUNCH();
        gm_while(q[2], q[3], mgs);
        depth = 4;
        k_gm_dot<<<grid(n, kRedThreads, kRedBlocks), kRedThreads, 0, q[3]>>>(B.V, B.w, n, B.st, B.a.hcol, B.partials,
                                                                              B.ticket, 0);
        FPB_CHECK_LAUNCH();
        k_gm_axpy<<<grid(n, 256, 4096), 256, 0, q[3]>>>(B.w, B.V, n, B.st, B.a.hcol);
        FPB_CHECK_LAUNCH();
        k_gm_mgs_next<<<1, 1, 0, q[3]>>>(B.st, mgs);
        FPB_CHECK_LAUNCH();
        cudaGraph_t junk = nullptr;
        FPB_CUDA(cudaStreamEndCapture(q[3], &junk));
        depth = 3;
        k_gm_dot<<<grid(n, kRedThreads, kRedBlocks), kRedThreads, 0, q[2]>>>(B.V, B.w, n, B.st, B.a.hcol, B.partials,
                                                                              B.ticket, 1);
        FPB_CHECK_LAUNCH();
        k_gm_next_basis<<<grid(n, 256, 4096), 256, 0, q[2]>>>(B.V, B.w, n, B.st, B.a.hcol);
        FPB_CHECK_LAUNCH();
        k_gm_arnoldi<<<1, 1, 0, q[2]>>>(B.st, B.a, m, inner);
        FPB_CHECK_LAUNCH();
        FPB_CUDA(cudaStreamEndCapture(q[2], &junk));
        depth = 2;
        k_gm_solve_y<<<1, 1, 0, q[1]>>>(B.st, B.a, m);
        FPB_CHECK_LAUNCH();
        k_gm_update<<<grid(n, 256, 4096), 256, 0, q[1]>>>(B.x, B.V, n, B.st, B.a.y);
        FPB_CHECK_LAUNCH();
        k_gm_outer_next<<<1, 1, 0, q[1]>>>(B.st, max_iter, outer);
        FPB_CHECK_LAUNCH();
        FPB_CUDA(cudaStreamEndCapture(q[1], &junk));
        depth = 1;
        FPB_CUDA(cudaStreamEndCapture(q[0], &g));
        depth = 0;
        note_launches(-(launches_noted() - before));  // captured, not run
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        g = nullptr;
        FPB_CUDA(e);
    }
    catch (...)
    {
        for (int k = depth - 1; k >= 0; --k)
        {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(q[k], &junk);
            if (k == 0 && junk) cudaGraphDestroy(junk);
        }
        note_launches(-(launches_noted() - before));
        for (auto& x : q) cudaStreamDestroy(x);
        throw;
    }
    for (auto& x : q) cudaStreamDestroy(x);
    return exec;
}
}  // namespace
}  // namespace fpb
