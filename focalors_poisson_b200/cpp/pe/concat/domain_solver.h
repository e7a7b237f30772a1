// Solver interfaces of the drop-in C++ layer (reference pe/concat/domain_solver.h:9-24).
#pragma once

#include "base/field/field2.h"
#include "base/field/field3.h"

class DomainSolver2D
{
public:
    DomainSolver2D() {}
    virtual ~DomainSolver2D() {}
    virtual void solve(field2& f) = 0;
};

class DomainSolver3D
{
public:
    DomainSolver3D() {}
    virtual ~DomainSolver3D() {}
    virtual void solve(field3& f) = 0;
};
