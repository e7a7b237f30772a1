// Test driver for the drop-in C++ interface: builds a composite geometry with the reference's own calls
// (Domain2DUniform, Geometry2D::connect/check/solve_prepare, Variable2D::set_center_field /
// set_boundary_type, ghost values written into Variable2D::buffer_map as the reference's boundary
// assembly reads them) and solves it with ConcatPoissonSolver2D.
//
//   composite_case <case file> [--tree-only]
//
// Case file (whitespace-separated text):
//   nd
//   nd lines:   nx ny hx hy bc_xneg bc_xpos bc_yneg bc_ypos        (PDEBoundaryType numbering)
//   nconn
//   nconn lines: a dir b                                           (Geometry2D::connect(a, dir, b))
//   m tol maxIter
//   nghost
//   nghost blocks: d face, then ny (x faces) or nx (y faces) values
//   then the right-hand side of each domain in order, row-major nx*ny
// Output: "root <index>", "level <k>: <indices>", and (without --tree-only) "field <d>" followed by its
// nx*ny solved values at full precision.
#include "base/domain/domain2d.h"
#include "base/domain/geometry2d.h"
#include "base/domain/variable2d.h"
#include "base/field/field2.h"
#include "pe/concat/concat_solver2d.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <vector>

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::cerr << "usage: composite_case <case file> [--tree-only]\n";
        return 2;
    }
    const bool    tree_only = argc > 2 && std::strcmp(argv[2], "--tree-only") == 0;
    std::ifstream in(argv[1]);
    if (!in)
    {
        std::cerr << "cannot open " << argv[1] << "\n";
        return 2;
    }
    try
    {
        int nd;
        in >> nd;
        std::vector<int>    nx(nd), ny(nd), bc(4 * nd);
        std::vector<double> hx(nd), hy(nd);
        // one allocation, so domain addresses ascend with the index (the root rule breaks ties by address)
        std::unique_ptr<Domain2DUniform[]> dom(new Domain2DUniform[nd]);
        Geometry2D                         geo;
        for (int d = 0; d < nd; ++d)
        {
            in >> nx[d] >> ny[d] >> hx[d] >> hy[d] >> bc[4 * d] >> bc[4 * d + 1] >> bc[4 * d + 2] >> bc[4 * d + 3];
            dom[d].name = "D" + std::to_string(d);
            dom[d].set_size(nx[d] * hx[d], ny[d] * hy[d]);
            dom[d].set_nx(nx[d]);
            dom[d].set_ny(ny[d]);
            geo.add_domain(&dom[d]);
        }
        int nconn;
        in >> nconn;
        for (int c = 0; c < nconn; ++c)
        {
            int a, dir, b;
            in >> a >> dir >> b;
            geo.connect(&dom[a], (LocationType)dir, &dom[b]);
        }
        for (int d = 0; d < nd; ++d) dom[d].set_spatial_step(hx[d], hy[d]);  // exact steps after connect
        geo.check();
        geo.solve_prepare();
        std::cout << "root " << geo.index_of(geo.tree_root) << "\n";
        for (size_t k = 0; k < geo.hierarchical_solve_levels.size(); ++k)
        {
            std::cout << "level " << k << ":";
            for (auto* d : geo.hierarchical_solve_levels[k]) std::cout << " " << geo.index_of(d);
            std::cout << "\n";
        }
        if (tree_only) return 0;

        int    m, max_iter;
        double tol;
        in >> m >> tol >> max_iter;

        Variable2D          v("u");
        std::vector<field2> fields(nd);
        v.set_geometry(geo);
        for (int d = 0; d < nd; ++d) v.set_center_field(&dom[d], fields[d]);
        for (int d = 0; d < nd; ++d)
            for (int f = 0; f < 4; ++f)
                if (bc[4 * d + f] != (int)PDEBoundaryType::Adjacented)
                    v.set_boundary_type(&dom[d], (LocationType)f, (PDEBoundaryType)bc[4 * d + f]);
        int nghost;
        in >> nghost;
        for (int g = 0; g < nghost; ++g)
        {
            int d, f;
            in >> d >> f;
            const int n   = f < 2 ? ny[d] : nx[d];
            double*   buf = v.buffer_map[&dom[d]][(LocationType)f];
            for (int k = 0; k < n; ++k) in >> buf[k];
        }
        for (int d = 0; d < nd; ++d)
            for (int i = 0; i < nx[d]; ++i)
                for (int j = 0; j < ny[d]; ++j) in >> fields[d](i, j);
        if (!in) throw std::runtime_error("case file truncated");

        ConcatPoissonSolver2D solver(&v);
        solver.set_parameter(m, tol, max_iter);
        solver.solve();
        for (int d = 0; d < nd; ++d)
        {
            std::cout << "field " << d << "\n";
            for (int k = 0; k < nx[d] * ny[d]; ++k) std::printf("%.17g\n", fields[d].value[k]);
        }
    }
    catch (const std::exception& e)
    {
        std::cout << "error: " << e.what() << std::endl;
        return 3;
    }
    return 0;
}
