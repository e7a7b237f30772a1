// Single-rectangle Poisson solver of the drop-in interface (reference pe/poisson/poisson_solver2d.h:10-34):
// same constructors and solve(field2&), computed on the GPU by libfpb200 (fp_rect_* in include/fp_capi.h).
#pragma once

#include "base/config.h"
#include "base/domain/domain2d.h"
#include "base/domain/variable2d.h"
#include "base/field/field2.h"
#include "base/location_boundary.h"
#include "instrumentor/timer.h"
#include "pe/concat/domain_solver.h"

#include <cmath>
#include <iostream>

struct fp_rect;

class PoissonSolver2D : public DomainSolver2D
{
public:
    PoissonSolver2D(int in_nx, int in_ny, double in_hx, double in_hy, PDEBoundaryType in_boundary_type_xneg,
                    PDEBoundaryType in_boundary_type_xpos, PDEBoundaryType in_boundary_type_yneg,
                    PDEBoundaryType in_boundary_type_ypos);
    PoissonSolver2D(Domain2DUniform* in_domain, Variable2D* in_variable = nullptr);
    ~PoissonSolver2D() override;
    PoissonSolver2D(const PoissonSolver2D&)            = delete;
    PoissonSolver2D& operator=(const PoissonSolver2D&) = delete;

    void solve(field2& f) override;

private:
    int      nx = 0, ny = 0;
    fp_rect* handle = nullptr;
};
