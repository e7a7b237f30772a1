// Device-resident PoissonSolver3D (pe/poisson/poisson_solver3d.cpp:49-123), used by the 3D rectangle entry
// points (fp_rect3d_*) and by the 3D composite solver.
#pragma once

#include "fp_internal.h"

#include <memory>

namespace fpb
{

struct DevRect3D
{
    int                                   nx = 0, ny = 0, nz = 0;
    std::unique_ptr<DevTransform<double>> tz, ty;
    std::unique_ptr<DevRect<double>>      chase;  // nz ny combined modes along x
    mutable DevBuf                        work, scratch;

    // bc: x-, x+, y-, y+, z-, z+ (PDEBoundaryType values; Adjacented faces act as Dirichlet)
    DevRect3D(int nx, int ny, int nz, double hx, double hy, double hz, const int* bc);
    // batch fields of nx * ny * nz values each (z contiguous), solved in place on stream s
    void solve(double* f, long long batch, cudaStream_t s) const;
    long long cells() const { return (long long)nx * ny * nz; }
};

}  // namespace fpb
