// Composite-geometry Poisson solver of the drop-in interface (reference pe/concat/concat_solver2d.h:18-56):
// same constructor, set_parameter and solve(), computed on the GPU by libfpb200 (fp_composite_* in
// include/fp_capi.h). solve() works in place on the Variable2D's fields, using its ghost buffers.
#pragma once

#include "base/config.h"
#include "base/domain/domain2d.h"
#include "base/domain/geometry2d.h"
#include "base/domain/geometry_tree.hpp"
#include "base/domain/variable2d.h"
#include "base/location_boundary.h"
#include "pe/concat/domain_solver.h"

#include <vector>

struct fp_composite;

class ConcatPoissonSolver2D
{
public:
    Variable2D* variable = nullptr;

    ConcatPoissonSolver2D() {}
    explicit ConcatPoissonSolver2D(Variable2D* in_variable);
    virtual ~ConcatPoissonSolver2D();
    ConcatPoissonSolver2D(const ConcatPoissonSolver2D&)            = delete;
    ConcatPoissonSolver2D& operator=(const ConcatPoissonSolver2D&) = delete;

    void set_parameter(int in_m, double in_tol, int in_maxIter);
    void solve();

protected:
    int    m       = 20;
    double tol     = 1e-8;
    int    maxIter = 100;

private:
    void                          construct();
    fp_composite*                 handle = nullptr;
    std::vector<Domain2DUniform*> order;
};
