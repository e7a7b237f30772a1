// PoissonSolver3D on the device (include/fp_capi.h fp_rect3d_*): the reference's 3D rectangle solve
// (pe/poisson/poisson_solver3d.cpp:49-123) with the kernels of the 2D solver. A field3 holds nx x ny x nz
// values, value(i, j, k) = f[(i ny + j) nz + k] (base/field/field3.cpp:378-388): z contiguous.
//
//   1. z-transform of the nx ny contiguous rows of length nz (the 2D y-transform kernel, family of the z pair)
//   2. per x-slab transpose (ny x nz -> nz x ny) into a work field laid out (i, k, j)
//   3. y-transform of the nx nz contiguous rows of length ny
//   4. partition chase along x: in the (i, k, j) layout row i holds every (z-mode k, y-mode j) pair
//      contiguously, so the 2D chase runs unchanged over ny nz "wavenumbers" with the diagonals
//      x_diag[k][j] = -2 + (hx/hy)^2 lambda_y[j] + (hx/hz)^2 lambda_z[k] (poisson_solver3d.cpp:57-70)
//   5. inverse y-transform, transpose back, inverse z-transform.
// The reference transposes the whole field three times to make each axis contiguous in turn; here only the
// y axis needs a transpose, because the chase reads its x-lines with one thread per mode (coalesced along
// the modes).
#include "../../include/fp_capi.h"
#include "fp_internal.h"
#include "fp_rect3d.h"

#include <cmath>
#include <memory>

namespace fpb
{
namespace
{
// Transposes nslab slabs of R x C doubles (row-major) into C x R, 32 x 32 tiles through shared memory.
__global__ void __launch_bounds__(256) k_slab_transpose(const double* __restrict__ in, double* __restrict__ out,
                                                        long long nslab, int R, int C)
{
    __shared__ double tile[32][33];
    const int         c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (long long sl = blockIdx.z; sl < nslab; sl += gridDim.z)
    {
        const double* a = in + sl * (long long)R * C;
        double*       o = out + sl * (long long)R * C;
        for (int dy = threadIdx.y; dy < 32; dy += 8)
        {
            const int r = r0 + dy, c = c0 + threadIdx.x;
            if (r < R && c < C) tile[dy][threadIdx.x] = a[(long long)r * C + c];
        }
        __syncthreads();
        for (int dy = threadIdx.y; dy < 32; dy += 8)
        {
            const int c = c0 + dy, r = r0 + threadIdx.x;
            if (r < R && c < C) o[(long long)c * R + r] = tile[threadIdx.x][dy];
        }
        __syncthreads();
    }
}

void slab_transpose(const double* in, double* out, long long nslab, int R, int C, cudaStream_t s)
{
    if (nslab <= 0) return;
    const dim3 grid((C + 31) / 32, (R + 31) / 32, (unsigned)std::min<long long>(nslab, 65535));
    k_slab_transpose<<<grid, dim3(32, 8), 0, s>>>(in, out, nslab, R, C);
    FPB_CHECK_LAUNCH();
}

// PoissonSolver3DBase::cal_lambda (pe/poisson/poisson_solver3d_base.cpp:41-74), i = 1..n, with the
// reference's own expressions.
std::vector<double> cal_lambda3(int n, int bn, int bp)
{
    const double        pi = 3.14159265358979323846;  // the reference's `pi` (base/pch.h:13)
    std::vector<double> lam(n);
    for (int i = 1; i <= n; ++i)
    {
        double v;
        if (bn == BC_PERIODIC && bp == BC_PERIODIC) v = -2.0 - 2.0 * std::cos(2.0 * pi / n * std::floor(i / 2.0));
        else if (bn == BC_NEUMANN && bp == BC_NEUMANN) v = -2.0 - 2.0 * std::cos(pi / n * i);
        else if (dir_like(bn) && dir_like(bp)) v = -2.0 + 2.0 * std::cos(pi / (n + 1) * i);
        else if ((dir_like(bn) && bp == BC_NEUMANN) || (bn == BC_NEUMANN && dir_like(bp)))
            v = -2.0 - 2.0 * std::cos(2.0 * pi * i / (2 * n + 1));
        else throw Error(FP_ERR_INVALID, "unsupported boundary pair");
        lam[i - 1] = v;
    }
    return lam;
}
}  // namespace

DevRect3D::DevRect3D(int nx_, int ny_, int nz_, double hx, double hy, double hz, const int* bc)
    : nx(nx_), ny(ny_), nz(nz_)
{
    if (nx < 2 || ny < 2 || nz < 2) throw Error(FP_ERR_INVALID, "each direction needs at least 2 cells");
    if (!(hx > 0) || !(hy > 0) || !(hz > 0)) throw Error(FP_ERR_INVALID, "grid spacings must be positive");
    const int ky = kind_of(bc[2], bc[3]), kz = kind_of(bc[4], bc[5]);
    if (ky < 0 || kz < 0) throw Error(FP_ERR_INVALID, "unsupported y or z boundary pair");
    tz.reset(new DevTransform<double>(kz, nz, true, true));
    ty.reset(new DevTransform<double>(ky, ny, true, true));
    const std::vector<double> ly = cal_lambda3(ny, bc[2], bc[3]), lz = cal_lambda3(nz, bc[4], bc[5]);
    std::vector<double>       d((size_t)ny * nz);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            d[(size_t)k * ny + j] = -2.0 + hx * hx / hy / hy * ly[j] + hx * hx / hz / hz * lz[k];
    bool no_dir = true;
    for (int f = 0; f < 6; ++f) no_dir = no_dir && !dir_like(bc[f]);
    const bool xp = bc[0] == BC_PERIODIC && bc[1] == BC_PERIODIC;
    // singular systems without a Dirichlet face (chasing_method3d.cpp:55-90): the last (k, j) pair, or
    // with periodic x every j of the last k
    const int sing_from = xp ? (nz - 1) * ny : nz * ny - 1;
    chase.reset(new DevRect<double>(nx, d, bc[0], bc[1], no_dir, sing_from));
}

void DevRect3D::solve(double* f, long long batch, cudaStream_t s) const
{
    if (batch <= 0) return;
    const long long n = (long long)nx * ny * nz;
    work.ensure((size_t)(batch * n) * sizeof(double));
    double* w = work.as<double>();
    tz->run(f, f, batch * nx * ny, false, s);
    slab_transpose(f, w, batch * nx, ny, nz, s);
    ty->run(w, w, batch * nx * nz, false, s);
    const long long need = chase->chase_scratch_elems(batch);
    if (need) scratch.ensure((size_t)need * sizeof(double));
    chase->chase(w, batch, scratch.as<double>(), s);
    ty->run(w, w, batch * nx * nz, true, s);
    slab_transpose(w, f, batch * nx, nz, ny, s);
    tz->run(f, f, batch * nx * ny, true, s);
}

}  // namespace fpb

struct fp_rect3d
{
    std::unique_ptr<fpb::DevRect3D> r;
    fpb::DevBuf                     staging;
};

using namespace fpb;

extern "C" {

int fp_rect3d_create(int nx, int ny, int nz, double hx, double hy, double hz, const int* bc, fp_rect3d** out)
{
    return guarded([&] {
        if (!out || !bc) throw Error(FP_ERR_INVALID, "null argument");
        *out = nullptr;
        require_device();
        std::unique_ptr<fp_rect3d> r(new fp_rect3d());
        r->r.reset(new DevRect3D(nx, ny, nz, hx, hy, hz, bc));
        *out = r.release();
    });
}

int fp_rect3d_solve_f64(fp_rect3d* r, double* f, long long batch, int flags, void* stream)
{
    return guarded([&] {
        if (!r || !r->r) throw Error(FP_ERR_INVALID, "null solver");
        if (!f) throw Error(FP_ERR_INVALID, "null field pointer");
        if (batch < 0) throw Error(FP_ERR_INVALID, "negative batch");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (flags & FP_DEVICE)
        {
            r->r->solve(f, batch, s);
            if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
            return;
        }
        const size_t bytes = (size_t)batch * r->r->nx * r->r->ny * r->r->nz * sizeof(double);
        r->staging.ensure(bytes);
        FPB_CUDA(cudaMemcpyAsync(r->staging.get(), f, bytes, cudaMemcpyHostToDevice, s));
        r->r->solve(r->staging.as<double>(), batch, s);
        FPB_CUDA(cudaMemcpyAsync(f, r->staging.get(), bytes, cudaMemcpyDeviceToHost, s));
        FPB_CUDA(cudaStreamSynchronize(s));
    });
}

int fp_rect3d_destroy(fp_rect3d* r)
{
    return guarded([&] { delete r; });
}

}  // extern "C"
