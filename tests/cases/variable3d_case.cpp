// A 3D case file in the reference's API (Geometry3D, Variable3D, ConcatPoissonSolver3D), compiled unchanged
// against the reference's own headers and sources and against the drop-in headers. Without arguments it
// prints the host bookkeeping (sizes propagated by connect, axis offsets, the tree, boundary types and their
// errors, set_value / set_buffer / set_boundary_value / set_corner results); with "solve" it solves the
// composite problem and prints the solution's sums and a few values.
#include "base/domain/domain3d.h"
#include "base/domain/geometry3d.h"
#include "base/domain/variable3d.h"
#include "base/field/field3.h"
#include "pe/concat/concat_solver3d.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

static double plane_sum(const field2& p)
{
    double s = 0;
    for (int i = 0; i < p.get_nx(); ++i)
        for (int j = 0; j < p.get_ny(); ++j) s += p(i, j);
    return s;
}

int main(int argc, char** argv)
{
    const bool solve = argc > 1 && std::string(argv[1]) == "solve";
    Domain3DUniform c(8, 6, 4, 1.0, 0.75, 0.5, "C");
    Domain3DUniform e("E"), u("U"), b("B");
    e.set_nx(5);
    e.set_lx(0.625);
    u.set_nz(3);
    u.set_lz(0.375);
    b.set_ny(4);
    b.set_ly(0.5);

    Geometry3D geo;
    geo.connect(&c, LocationType::XPositive, &e);
    geo.connect(&c, LocationType::ZPositive, &u);
    geo.connect(&e, LocationType::YNegative, &b);
    geo.check();
    geo.solve_prepare();
    geo.axis(&c, LocationType::XNegative);
    geo.axis(&c, LocationType::YNegative);
    geo.axis(&c, LocationType::ZNegative);

    std::vector<Domain3DUniform*> all = {&c, &e, &u, &b};
    if (!solve)
    {
        for (auto* d : all)
            std::printf("%s n %d %d %d l %.17g %.17g %.17g h %.17g %.17g %.17g o %.17g %.17g %.17g\n", d->name.c_str(),
                        d->nx, d->ny, d->nz, d->lx, d->ly, d->lz, d->hx, d->hy, d->hz, d->get_offset_x(),
                        d->get_offset_y(), d->get_offset_z());
        std::printf("root %s\n", geo.tree_root->name.c_str());
        for (size_t l = 0; l < geo.hierarchical_solve_levels.size(); ++l)
            for (auto* d : geo.hierarchical_solve_levels[l]) std::printf("level %zu %s\n", l, d->name.c_str());
        for (auto* d : all)
            if (geo.parent_map.count(d))
                std::printf("parent %s %d %s\n", d->name.c_str(), (int)geo.parent_map[d].first,
                            geo.parent_map[d].second->name.c_str());
    }

    Variable3D v("p");
    v.set_geometry(geo);
    field3 fc, fe, fu, fb;
    v.set_center_field(&c, fc);
    v.set_center_field(&e, fe);
    v.set_center_field(&u, fu);
    v.set_center_field(&b, fb);
    v.set_boundary_type(&c, LocationType::XNegative, PDEBoundaryType::Neumann);
    v.set_boundary_type(&b, LocationType::YNegative, PDEBoundaryType::Neumann);
    v.set_boundary_type(&u, {{LocationType::ZPositive, PDEBoundaryType::Neumann}});
    try
    {
        v.set_boundary_type(&c, LocationType::XPositive, PDEBoundaryType::Dirichlet);
    }
    catch (const std::exception& ex)
    {
        if (!solve) std::printf("error: %s\n", ex.what());
    }
    v.set_boundary_type(PDEBoundaryType::Dirichlet);
    if (!solve)
        for (auto* d : all)
        {
            std::printf("types %s", d->name.c_str());
            for (int f = 0; f < 6; ++f) std::printf(" %d", (int)v.boundary_type_map[d][(LocationType)f]);
            std::printf("\n");
        }

    auto rhs = [](double x, double y, double z) { return std::sin(3.0 * x + 1.0) * std::cos(2.0 * y) + z * z - 0.5 * x * y; };
    auto gh  = [](double x, double y, double z) { return 0.25 * x - 0.5 * y + z + 0.125; };
    v.set_value(rhs);
    v.set_buffer(gh);
    if (!solve)
    {
        for (auto* d : all)
        {
            std::printf("field %s %.17g %.17g %.17g\n", d->name.c_str(), v.field_map[d]->sum(), v.field_map[d]->norm(),
                        (*v.field_map[d])(d->nx - 1, 0, d->nz - 1));
            for (int f = 0; f < 6; ++f) std::printf("buffer %s %d %.17g\n", d->name.c_str(), f, plane_sum(*v.buffer_map[d][(LocationType)f]));
        }
        v.set_boundary_value(&c, LocationType::YPositive, 2.5);
        v.set_boundary_value(&u, LocationType::ZPositive, gh);
        std::printf("bvalue %.17g %.17g\n", plane_sum(*v.boundary_value_map[&c][LocationType::YPositive]),
                    plane_sum(*v.boundary_value_map[&u][LocationType::ZPositive]));
        Variable3D w("w");
        w.set_geometry(geo);
        field3 x1;
        w.set_x_face_center_field(&c, x1);
        w.set_corner(&c, gh);
        double cy = 0, cz = 0;
        for (int j = 0; j < c.ny; ++j) cy += w.corner_y_map[&c][j];
        for (int k = 0; k < c.nz; ++k) cz += w.corner_z_map[&c][k];
        std::printf("corner %.17g %.17g\n", cy, cz);
        return 0;
    }

    ConcatPoissonSolver3D solver(&v);
    solver.set_parameter(20, 1e-13, 100);
    solver.solve();
    for (auto* d : all)
        std::printf("solution %s %.17g %.17g %.17g %.17g\n", d->name.c_str(), v.field_map[d]->sum(),
                    v.field_map[d]->norm(), (*v.field_map[d])(0, 0, 0), (*v.field_map[d])(d->nx - 1, d->ny - 1, d->nz - 1));
    return 0;
}
