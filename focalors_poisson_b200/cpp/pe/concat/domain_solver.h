// Solver interface of the drop-in C++ layer (reference pe/concat/domain_solver.h:9-15).
#pragma once

#include "base/field/field2.h"

class DomainSolver2D
{
public:
    DomainSolver2D() {}
    virtual ~DomainSolver2D() {}
    virtual void solve(field2& f) = 0;
};
