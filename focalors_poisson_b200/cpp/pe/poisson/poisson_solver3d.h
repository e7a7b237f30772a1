// Single-box Poisson solver of the drop-in interface (reference pe/poisson/poisson_solver3d.h:9-41):
// PoissonSolver3D on the GPU through fp_rect3d_* (include/fp_capi.h).
#pragma once

#include "base/config.h"
#include "base/domain/domain3d.h"
#include "base/domain/variable3d.h"
#include "base/field/field3.h"
#include "pe/concat/domain_solver.h"

struct fp_rect3d;

class PoissonSolver3D : public DomainSolver3D
{
public:
    PoissonSolver3D() {}
    PoissonSolver3D(int in_nx, int in_ny, int in_nz, double in_hx, double in_hy, double in_hz,
                    PDEBoundaryType in_boundary_type_xneg, PDEBoundaryType in_boundary_type_xpos,
                    PDEBoundaryType in_boundary_type_yneg, PDEBoundaryType in_boundary_type_ypos,
                    PDEBoundaryType in_boundary_type_zneg, PDEBoundaryType in_boundary_type_zpos);
    PoissonSolver3D(Domain3DUniform* in_domain, Variable3D* in_variable = nullptr);
    ~PoissonSolver3D() override;
    PoissonSolver3D(const PoissonSolver3D&)            = delete;
    PoissonSolver3D& operator=(const PoissonSolver3D&) = delete;

    void solve(field3& f) override;

private:
    int        nx = 0, ny = 0, nz = 0;
    fp_rect3d* handle = nullptr;
};
