// Host data-model driver: builds a composite geometry with the reference's user API (Domain2DUniform,
// Geometry2D::connect / axis / check / solve_prepare, Variable2D::set_geometry / set_*_field /
// set_boundary_type / set_buffer / set_value / set_boundary_value / set_boundary / set_corner) and prints
// what that API leaves behind: domain sizes, steps and offsets, the tree root, boundary types, field
// values, ghost buffers, boundary values and corner values, for centre, x-edge, y-edge and corner fields.
// Compiled once against the reference's headers and sources and once against the drop-in headers, the
// two outputs must be equal.
#include "base/domain/domain2d.h"
#include "base/domain/geometry2d.h"
#include "base/domain/variable2d.h"
#include "base/field/field2.h"

#include <cmath>
#include <cstdio>
#include <vector>

int main()
{
    Geometry2D      geo;
    Domain2DUniform C(8, 6, 1.0, 0.75, "C");
    Domain2DUniform W("W"), E("E"), S("S"), N("N");
    W.set_nx(4);
    W.set_lx(0.5);
    E.set_nx(6);
    E.set_lx(0.75);
    S.set_ny(5);
    S.set_ly(0.5);
    N.set_ny(3);
    N.set_ly(0.25);
    geo.add_domain({&C, &W, &E, &S, &N});
    geo.connect(&C, LocationType::XNegative, &W);
    geo.connect(&C, LocationType::XPositive, &E);
    geo.connect(&C, LocationType::YNegative, &S);
    geo.connect(&C, LocationType::YPositive, &N);
    geo.check();
    geo.solve_prepare();
    geo.axis(&W, LocationType::XNegative);
    geo.axis(&S, LocationType::YNegative);

    Variable2D v("v");
    v.set_geometry(geo);
    std::vector<Domain2DUniform*> doms = {&C, &W, &E, &S, &N};
    std::vector<field2>           f(doms.size());
    for (size_t d = 0; d < doms.size(); ++d) v.set_center_field(doms[d], f[d]);
    v.set_boundary_type(&W, LocationType::XNegative, PDEBoundaryType::Neumann);
    v.set_boundary_type(&N, {{LocationType::YPositive, PDEBoundaryType::Neumann}});
    v.set_boundary_type(PDEBoundaryType::Dirichlet);
    v.set_value([](double x, double y) { return std::sin(3.0 * x) * std::cos(2.0 * y) + x * y; });
    v.set_buffer([](double x, double y) { return x * x - 0.5 * y + 1.0; });

    std::printf("root %s\n", geo.tree_root->name.c_str());
    const LocationType faces[4] = {LocationType::XNegative, LocationType::XPositive, LocationType::YNegative,
                                   LocationType::YPositive};
    for (size_t d = 0; d < doms.size(); ++d)
    {
        Domain2DUniform* s = doms[d];
        std::printf("domain %s %d %d %.17g %.17g %.17g %.17g\n", s->name.c_str(), s->get_nx(), s->get_ny(),
                    s->get_hx(), s->get_hy(), s->get_offset_x(), s->get_offset_y());
        for (int k = 0; k < 4; ++k) std::printf(" bc%d %d", k, (int)v.boundary_type_map[s][faces[k]]);
        std::printf("\n");
        for (int i = 0; i < f[d].get_nx(); ++i)
            for (int j = 0; j < f[d].get_ny(); ++j) std::printf("%.17g\n", f[d](i, j));
        for (int k = 0; k < 4; ++k)
        {
            const int n   = k < 2 ? s->get_ny() : s->get_nx();
            double*   buf = v.buffer_map[s][faces[k]];
            std::printf("buffer %d\n", k);
            for (int q = 0; q < n && buf; ++q) std::printf("%.17g\n", buf[q]);
        }
    }

    // boundary values, corners and the staggered positions (x-edge, y-edge, node-centred corner fields)
    v.set_boundary_value(&C, LocationType::YNegative, 2.5);
    v.set_boundary_value(&E, LocationType::XPositive, [](double x, double y) { return x - 3.0 * y; });
    v.set_boundary([](double x, double y) { return std::cos(x + 2.0 * y); });
    for (size_t d = 0; d < doms.size(); ++d)
        for (int k = 0; k < 4; ++k)
        {
            Domain2DUniform* s = doms[d];
            if (!v.has_boundary_value_map[s][faces[k]]) continue;
            const int n = k < 2 ? s->get_ny() : s->get_nx();
            std::printf("boundary value %s %d\n", s->name.c_str(), k);
            for (int q = 0; q < n; ++q) std::printf("%.17g\n", v.boundary_value_map[s][faces[k]][q]);
        }
    std::printf("corner C %.17g\n", v.xpos_yneg_corner_map[&C]);
    const char* kinds[3] = {"xedge", "yedge", "corner"};
    for (int kind = 0; kind < 3; ++kind)
    {
        Variable2D          w(kinds[kind]);
        std::vector<field2> g(doms.size());
        w.set_geometry(geo);
        for (size_t d = 0; d < doms.size(); ++d)
        {
            if (kind == 0) w.set_x_edge_field(doms[d], g[d]);
            else if (kind == 1) w.set_y_edge_field(doms[d], g[d]);
            else w.set_corner_field(doms[d], g[d]);
        }
        w.set_boundary_type(PDEBoundaryType::Dirichlet);
        w.set_value([](double x, double y) { return x * x + 0.25 * y; });
        w.set_buffer([](double x, double y) { return 2.0 * x - y; });
        w.set_boundary([](double x, double y) { return x * y + 1.0; });
        w.set_corner([](double x, double y) { return x + 10.0 * y; });
        for (size_t d = 0; d < doms.size(); ++d)
        {
            Domain2DUniform* s = doms[d];
            std::printf("%s %s %d %d %d\n", kinds[kind], s->name.c_str(), g[d].get_nx(), g[d].get_ny(),
                        (int)w.position_type);
            for (int i = 0; i < g[d].get_nx(); ++i)
                for (int j = 0; j < g[d].get_ny(); ++j) std::printf("%.17g\n", g[d](i, j));
            const int extra = kind == 2 ? 1 : 0;
            for (int k = 0; k < 4; ++k)
            {
                const int n = (k < 2 ? s->get_ny() : s->get_nx()) + extra;
                std::printf("buffer %d\n", k);
                for (int q = 0; q < n; ++q) std::printf("%.17g\n", w.buffer_map[s][faces[k]][q]);
                if (!w.has_boundary_value_map[s][faces[k]]) continue;
                std::printf("boundary value %d\n", k);
                for (int q = 0; q < n; ++q) std::printf("%.17g\n", w.boundary_value_map[s][faces[k]][q]);
            }
            if (w.xpos_yneg_corner_map.count(s)) std::printf("corner xpos_yneg %.17g\n", w.xpos_yneg_corner_map[s]);
            if (w.xneg_ypos_corner_map.count(s)) std::printf("corner xneg_ypos %.17g\n", w.xneg_ypos_corner_map[s]);
        }
    }
    return 0;
}
