// 3D composite-geometry Poisson solver of the drop-in interface (reference pe/concat/concat_solver3d.h:18-54):
// same constructor, set_parameter and solve(), computed on the GPU by libfpb200 (fp_composite3d_* in
// include/fp_capi.h). solve() works in place on the Variable3D's fields, using its ghost planes.
#pragma once

#include "base/config.h"
#include "base/domain/domain3d.h"
#include "base/domain/geometry3d.h"
#include "base/domain/geometry_tree.hpp"
#include "base/domain/variable3d.h"
#include "base/location_boundary.h"
#include "pe/concat/domain_solver.h"

#include <vector>

struct fp_composite3d;

class ConcatPoissonSolver3D
{
public:
    Variable3D* variable = nullptr;

    explicit ConcatPoissonSolver3D(Variable3D* in_variable);
    ~ConcatPoissonSolver3D();
    ConcatPoissonSolver3D(const ConcatPoissonSolver3D&)            = delete;
    ConcatPoissonSolver3D& operator=(const ConcatPoissonSolver3D&) = delete;

    void set_parameter(int in_m, double in_tol, int in_maxIter);
    void solve();

private:
    void                          construct();
    fp_composite3d*               handle = nullptr;
    std::vector<Domain3DUniform*> order;
    int                           m       = 20;
    double                        tol     = 1e-8;
    int                           maxIter = 100;
};
