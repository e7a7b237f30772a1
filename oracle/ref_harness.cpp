// C entry points over the reference's own serial 2D Poisson path, compiled from the reference's
// unmodified sources into oracle/_ref/libfpref.so by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY. Used to generate the golden fixtures in tests/golden/, to pin the numpy
// restatement in oracle/fp_oracle.py, and as the timed CPU baseline ("reference" arm of bench.py).
// It is never part of the product path.
//
// Entry points and the reference code each one drives:
//   fpref_transform       PoissonFFT2D_{DD,NN,ND,DN,PP}::transform / transform_transpose
//                         (pe/poisson/poisson_fft2d.cpp:19-465), chosen like
//                         PoissonSolver2DBase::create_fft (pe/poisson/poisson_solver2d_base.cpp:64-91)
//   fpref_poisson2d_solve PoissonSolver2D(nx,ny,hx,hy,4 x BC).solve (pe/poisson/poisson_solver2d.cpp:3-90)
//   fpref_poisson3d_solve PoissonSolver3D(nx,ny,nz,hx,hy,hz,6 x BC).solve
//                         (pe/poisson/poisson_solver3d.cpp:3-123)
//   fpref_concat_*        Geometry2D + Variable2D + ConcatPoissonSolver2D
//                         (pe/concat/concat_solver2d.cpp:19-223), the case-file flow of
//                         case/validation/2d/concat_solver_reference.cpp:42-115
//   fpref_concat3d_*      Geometry3D + Variable3D + ConcatPoissonSolver3D
//                         (pe/concat/concat_solver3d.cpp:5-247)
//   fpref_add_random      add_random_number(field2&, ...) (base/math/random.cpp:24-46)
//   fpref_gmres_mock / fpref_schur_mock
//                         GMRESSolver2D / SchurMat2D_* with the mock branch solver of
//                         case/validation/2d/gmres_reference.cpp:8-23 and shur_mat_reference.cpp:6-21
#include "base/pch.h"

#include "base/domain/domain2d.h"
#include "base/domain/geometry2d.h"
#include "base/domain/variable2d.h"
#include "base/math/random.h"
#include "base/domain/domain3d.h"
#include "base/domain/geometry3d.h"
#include "base/domain/variable3d.h"
#include "pe/concat/concat_solver2d.h"
#include "pe/concat/concat_solver3d.h"
#include "pe/concat/gmres_solver2d.h"
#include "pe/concat/schur_mat2d.h"
#include "pe/poisson/poisson_fft2d.h"
#include "pe/poisson/poisson_solver2d.h"
#include "pe/poisson/poisson_solver3d.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

namespace
{
PDEBoundaryType bc_of(int v) { return static_cast<PDEBoundaryType>(v); }
LocationType    loc_of(int v) { return static_cast<LocationType>(v); }

void copy_in(field2& f, const double* src)
{
    for (int i = 0; i < f.get_nx(); ++i)
        for (int j = 0; j < f.get_ny(); ++j) f(i, j) = src[(size_t)i * f.get_ny() + j];
}
void copy_out(const field2& f, double* dst)
{
    for (int i = 0; i < f.get_nx(); ++i)
        for (int j = 0; j < f.get_ny(); ++j) dst[(size_t)i * f.get_ny() + j] = f(i, j);
}

// Mock branch solver of case/validation/2d/gmres_reference.cpp:8-23: f(i,j) *= i*ny + j + 1.
class MockSolver : public DomainSolver2D
{
public:
    void solve(field2& f) override
    {
        for (int i = 0; i < f.get_nx(); i++)
            for (int j = 0; j < f.get_ny(); j++) f(i, j) *= i * f.get_ny() + j + 1;
    }
};

// Branch solver that answers a Schur construction's unit-impulse solves from a supplied dense
// interface matrix S (S[j*cn+i] = response at interface cell j to an impulse at cell i), so that
// the CPU baseline can be set up at sizes where the reference's own cn-solve construction
// (pe/concat/schur_mat2d.cpp:5-106) would take hours. Only the interface row/column is written,
// which is all SchurMat2D_*::construct reads.
class MatrixBranchSolver : public DomainSolver2D
{
public:
    MatrixBranchSolver(LocationType loc_from_parent, const double* S, int cn)
        : loc(loc_from_parent), S(S), cn(cn)
    {}
    void solve(field2& t) override
    {
        const int bnx = t.get_nx(), bny = t.get_ny();
        int       src = -1;
        for (int i = 0; i < cn && src < 0; ++i)
        {
            double v = 0;
            switch (loc)
            {
                case LocationType::XNegative: v = t(bnx - 1, i); break;
                case LocationType::XPositive: v = t(0, i); break;
                case LocationType::YPositive: v = t(i, 0); break;
                case LocationType::YNegative: v = t(i, bny - 1); break;
                default: break;
            }
            if (v == 1.0) src = i;
        }
        t.clear(0.0);
        if (src < 0) return;
        for (int j = 0; j < cn; ++j)
        {
            const double v = S[(size_t)j * cn + src];
            switch (loc)
            {
                case LocationType::XNegative: t(bnx - 1, j) = v; break;
                case LocationType::XPositive: t(0, j) = v; break;
                case LocationType::YPositive: t(j, 0) = v; break;
                case LocationType::YNegative: t(j, bny - 1) = v; break;
                default: break;
            }
        }
    }

private:
    LocationType  loc;
    const double* S;
    int           cn;
};

// ConcatPoissonSolver2D with the GMRES parameters fixed before the one and only construction
// (the public set_parameter would construct twice: concat_solver2d.cpp:7-17).
class HarnessConcat : public ConcatPoissonSolver2D
{
public:
    HarnessConcat(Variable2D* v, int m_, double tol_, int maxIter_, bool construct)
    {
        variable = v;
        m        = m_;
        tol      = tol_;
        maxIter  = maxIter_;
        init_before_constructing_solver(variable);
        if (construct) construct_solver_map();
    }
    // Root-only injection: leaves get the reference's PoissonSolver2D; the root GMRES gets its
    // Schur matrices from MatrixBranchSolver columns. Valid when every child of the root is a leaf.
    bool construct_with_matrices(const std::vector<const double*>& S_by_domain, Geometry2D& geo)
    {
        for (auto* d : geo.domains)
            if (d != tree_root && !tree_map[d].empty()) return false;
        for (auto* d : geo.domains)
            if (d != tree_root) solver_map[d] = new PoissonSolver2D(d, variable);
        std::unordered_map<Domain2DUniform*, DomainSolver2D*> fake;
        std::vector<std::unique_ptr<MatrixBranchSolver>>      keep;
        for (auto& [loc, child] : tree_map[tree_root])
        {
            size_t idx = std::find(geo.domains.begin(), geo.domains.end(), child) - geo.domains.begin();
            int    cn  = (loc == LocationType::XNegative || loc == LocationType::XPositive) ? child->ny : child->nx;
            keep.emplace_back(new MatrixBranchSolver(loc, S_by_domain[idx], cn));
            fake[child] = keep.back().get();
        }
        auto* gmres               = new GMRESSolver2D(tree_root, m, tol, maxIter);
        gmres->set_solver(new PoissonSolver2D(tree_root, variable));
        gmres->schur_mat_construct(tree_map[tree_root], fake);
        solver_map[tree_root] = gmres;
        return true;
    }
    Domain2DUniform* root() const { return tree_root; }
    const std::vector<std::vector<Domain2DUniform*>>& levels() const { return hierarchical_solve_levels; }
};

struct ConcatCase
{
    std::vector<Domain2DUniform>      domains;
    Geometry2D                        geo;
    std::unique_ptr<Variable2D>       var;
    std::vector<field2>               fields;
    std::unique_ptr<HarnessConcat>    solver;
    std::vector<int>                  nx, ny;
    double                            t_construct = 0.0;
};
}  // namespace

extern "C" {

// Forward (inverse == 0) or transpose (inverse != 0) y-transform of an nx x ny row-major field.
int fpref_transform(int bc_neg, int bc_pos, int nx, int ny, int inverse, const double* in, double* out)
{
    PDEBoundaryType n = bc_of(bc_neg), p = bc_of(bc_pos);
    PoissonFFT2D*   fft = nullptr;
    if (n == PDEBoundaryType::Periodic && p == PDEBoundaryType::Periodic) fft = new PoissonFFT2D_PP();
    else if (n == PDEBoundaryType::Neumann && p == PDEBoundaryType::Neumann) fft = new PoissonFFT2D_NN();
    else if (isDirLike(n) && isDirLike(p)) fft = new PoissonFFT2D_DD();
    else if (isDirLike(n) && p == PDEBoundaryType::Neumann) fft = new PoissonFFT2D_DN();
    else if (n == PDEBoundaryType::Neumann && isDirLike(p)) fft = new PoissonFFT2D_ND();
    else return 1;
    fft->init(nx, ny);
    field2 a(nx, ny), b(nx, ny);
    copy_in(a, in);
    if (inverse) fft->transform_transpose(a, b);
    else fft->transform(a, b);
    copy_out(b, out);
    delete fft;
    return 0;
}

// PoissonSolver2D(nx, ny, hx, hy, bc[0..3]).solve(f), f row-major nx x ny, in place.
// bc order: XNegative, XPositive, YNegative, YPositive (PDEBoundaryType values).
int fpref_poisson2d_solve(int nx, int ny, double hx, double hy, const int* bc, double* f, int repeats,
                          double* seconds_per_solve)
{
    PoissonSolver2D s(nx, ny, hx, hy, bc_of(bc[0]), bc_of(bc[1]), bc_of(bc[2]), bc_of(bc[3]));
    field2          F(nx, ny);
    std::vector<double> keep(f, f + (size_t)nx * ny);
    if (repeats < 1) repeats = 1;
    std::vector<double> times;
    for (int r = 0; r < repeats; ++r)
    {
        copy_in(F, keep.data());
        auto t0 = std::chrono::steady_clock::now();
        s.solve(F);
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    copy_out(F, f);
    if (seconds_per_solve)
    {
        std::sort(times.begin(), times.end());
        *seconds_per_solve = times[times.size() / 2];
    }
    return 0;
}

// PoissonSolver3D on a field3 of nx x ny x nz values, value(i, j, k) = f[(i ny + j) nz + k]
// (base/field/field3.cpp:378-388); bc in the order x-, x+, y-, y+, z-, z+.
int fpref_poisson3d_solve(int nx, int ny, int nz, double hx, double hy, double hz, const int* bc, double* f,
                          int repeats, double* seconds_per_solve)
{
    PoissonSolver3D s(nx, ny, nz, hx, hy, hz, bc_of(bc[0]), bc_of(bc[1]), bc_of(bc[2]), bc_of(bc[3]), bc_of(bc[4]),
                      bc_of(bc[5]));
    const size_t        n = (size_t)nx * ny * nz;
    std::vector<double> keep(f, f + n), times;
    field3              F(nx, ny, nz);
    if (repeats < 1) repeats = 1;
    for (int r = 0; r < repeats; ++r)
    {
        F.set_size(nx, ny, nz);
        std::memcpy(F.value, keep.data(), n * sizeof(double));
        auto t0 = std::chrono::steady_clock::now();
        s.solve(F);
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    std::memcpy(f, F.value, n * sizeof(double));
    if (seconds_per_solve)
    {
        std::sort(times.begin(), times.end());
        *seconds_per_solve = times[times.size() / 2];
    }
    return 0;
}

// Build a composite case: domains[i] = Domain2DUniform(nx[i], ny[i], lx[i], ly[i]) allocated
// contiguously in index order (so the reference's address tie-break in TreeUtils::findOptimalRoot,
// base/domain/geometry_tree.hpp:84-93, picks the lower index); connect(a[k], dir[k], b[k]) in order;
// every non-adjacented face gets bc[4*i + face]. Schur construction happens here (timed) unless
// S_inject is non-null, in which case the root's Schur matrices are taken from S_inject[i] (one per
// child domain index i, row-major cn x cn; NULL for non-children).
void* fpref_concat_create(int nd, const int* nx, const int* ny, const double* lx, const double* ly, int nc,
                          const int* ca, const int* cdir, const int* cb, const int* bc, int m, double tol,
                          int maxIter, const double* const* S_inject)
{
    auto* c = new ConcatCase();
    c->domains.reserve(nd);
    for (int i = 0; i < nd; ++i)
        c->domains.emplace_back(nx[i], ny[i], lx[i], ly[i], "D" + std::to_string(i));
    for (int i = 0; i < nd; ++i) c->geo.add_domain(&c->domains[i]);
    for (int k = 0; k < nc; ++k) c->geo.connect(&c->domains[ca[k]], loc_of(cdir[k]), &c->domains[cb[k]]);
    c->geo.check();
    c->geo.solve_prepare();
    c->var.reset(new Variable2D("v"));
    c->var->set_geometry(c->geo);
    c->fields.resize(nd);
    for (int i = 0; i < nd; ++i) c->var->set_center_field(&c->domains[i], c->fields[i]);
    for (int i = 0; i < nd; ++i)
        for (int f = 0; f < 4; ++f)
        {
            auto& tm = c->var->boundary_type_map[&c->domains[i]];
            if (tm.count(loc_of(f)) && tm[loc_of(f)] == PDEBoundaryType::Adjacented) continue;
            c->var->set_boundary_type(&c->domains[i], loc_of(f), bc_of(bc[4 * i + f]));
        }
    for (int i = 0; i < nd; ++i)
    {
        c->nx.push_back(c->domains[i].nx);
        c->ny.push_back(c->domains[i].ny);
    }
    auto t0 = std::chrono::steady_clock::now();
    if (S_inject)
    {
        c->solver.reset(new HarnessConcat(c->var.get(), m, tol, maxIter, false));
        std::vector<const double*> S(S_inject, S_inject + nd);
        if (!c->solver->construct_with_matrices(S, c->geo))
        {
            delete c;
            return nullptr;
        }
    }
    else
    {
        c->solver.reset(new HarnessConcat(c->var.get(), m, tol, maxIter, true));
    }
    auto t1        = std::chrono::steady_clock::now();
    c->t_construct = std::chrono::duration<double>(t1 - t0).count();
    return c;
}

double fpref_concat_construct_seconds(void* h) { return static_cast<ConcatCase*>(h)->t_construct; }

// Index of the tree root and the BFS level of every domain (root = 0).
int fpref_concat_tree(void* h, int* root, int* level_of)
{
    auto* c = static_cast<ConcatCase*>(h);
    for (size_t i = 0; i < c->domains.size(); ++i)
        if (&c->domains[i] == c->geo.tree_root) *root = (int)i;
    for (size_t l = 0; l < c->geo.hierarchical_solve_levels.size(); ++l)
        for (auto* d : c->geo.hierarchical_solve_levels[l]) level_of[d - c->domains.data()] = (int)l;
    return 0;
}

// Fill fields (RHS) and ghost buffers, run ConcatPoissonSolver2D::solve `repeats` times (re-filling
// the inputs before each, because solve() mutates them), copy the last solution out. ghosts holds
// 4*nd pointers (XNeg, XPos, YNeg, YPos per domain; NULL = zero). Returns the median solve time.
double fpref_concat_solve(void* h, const double* const* rhs, const double* const* ghosts, double* const* out,
                          int repeats)
{
    auto* c  = static_cast<ConcatCase*>(h);
    int   nd = (int)c->domains.size();
    if (repeats < 1) repeats = 1;
    std::vector<double> times;
    for (int r = 0; r < repeats; ++r)
    {
        for (int i = 0; i < nd; ++i)
        {
            copy_in(c->fields[i], rhs[i]);
            for (int f = 0; f < 4; ++f)
            {
                double* buf = c->var->buffer_map[&c->domains[i]][loc_of(f)];
                int     len = (f < 2) ? c->ny[i] : c->nx[i];
                for (int k = 0; k < len; ++k) buf[k] = (ghosts && ghosts[4 * i + f]) ? ghosts[4 * i + f][k] : 0.0;
            }
        }
        auto t0 = std::chrono::steady_clock::now();
        c->solver->solve();
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    for (int i = 0; i < nd; ++i) copy_out(c->fields[i], out[i]);
    std::sort(times.begin(), times.end());
    return times[times.size() / 2];
}

void fpref_concat_destroy(void* h) { delete static_cast<ConcatCase*>(h); }

// case/validation/2d/gmres_reference.cpp:25-72 for one neighbour direction `loc`:
// root nx x ny, neighbour size n along the connection axis, mock solver, GMRES(m, tol, maxIter)
// on p_root(i,j) = i*ny + j + 1. Writes the result (nx*ny) to out.
int fpref_gmres_mock(int loc, int nx, int ny, int neighbor_n, int m, double tol, int maxIter, double* out)
{
    int neighbor_nx = nx, neighbor_ny = ny;
    if (loc_of(loc) == LocationType::XNegative || loc_of(loc) == LocationType::XPositive) neighbor_nx = neighbor_n;
    else neighbor_ny = neighbor_n;
    Domain2DUniform root(nx, ny, "root");
    Domain2DUniform neighbor(neighbor_nx, neighbor_ny, "neighbor");
    field2          p_root(nx, ny, "p_root");
    GMRESSolver2D   gmres(&root, m, tol, maxIter);
    MockSolver*     test_solver = new MockSolver();
    gmres.set_solver(test_solver);
    std::unordered_map<LocationType, Domain2DUniform*> adj;
    adj[loc_of(loc)] = &neighbor;
    std::unordered_map<Domain2DUniform*, DomainSolver2D*> solver_map;
    solver_map[&root]     = &gmres;
    solver_map[&neighbor] = test_solver;
    gmres.schur_mat_construct(adj, solver_map);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) p_root(i, j) = i * ny + j + 1;
    gmres.solve(p_root);
    copy_out(p_root, out);
    return 0;
}

// case/validation/2d/shur_mat_reference.cpp:23-66 for one direction: neighbour domain
// (bnx, bny), mock solver, f(i,j) = i*ny + j + 1 on an nx x ny root; writes S (cn*cn) and S*f (nx*ny).
int fpref_schur_mock(int loc, int bnx, int bny, int nx, int ny, double* S_out, double* prod_out)
{
    Domain2DUniform nb(bnx, bny, "nb");
    std::unique_ptr<SchurMat2D> S;
    switch (loc_of(loc))
    {
        case LocationType::XNegative: S.reset(new SchurMat2D_xneg(&nb)); break;
        case LocationType::XPositive: S.reset(new SchurMat2D_xpos(&nb)); break;
        case LocationType::YPositive: S.reset(new SchurMat2D_ypos(&nb)); break;
        case LocationType::YNegative: S.reset(new SchurMat2D_yneg(&nb)); break;
        default: return 1;
    }
    MockSolver solver;
    S->construct(&solver);
    field2 f(nx, ny);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) f(i, j) = i * ny + j + 1;
    field2 r  = (*S) * f;
    int    cn = S->get_size();
    // S->value is protected; recover it column by column through operator* on unit root edges.
    for (int i = 0; i < cn; ++i)
    {
        field2 e(nx, ny);
        switch (loc_of(loc))
        {
            case LocationType::XNegative: e(0, i) = 1.0; break;
            case LocationType::XPositive: e(nx - 1, i) = 1.0; break;
            case LocationType::YPositive: e(i, ny - 1) = 1.0; break;
            case LocationType::YNegative: e(i, 0) = 1.0; break;
            default: break;
        }
        field2 col = (*S) * e;
        for (int j = 0; j < cn; ++j)
        {
            double v = 0;
            switch (loc_of(loc))
            {
                case LocationType::XNegative: v = col(0, j); break;
                case LocationType::XPositive: v = col(nx - 1, j); break;
                case LocationType::YPositive: v = col(j, ny - 1); break;
                case LocationType::YNegative: v = col(j, 0); break;
                default: break;
            }
            S_out[(size_t)j * cn + i] = v;
        }
    }
    copy_out(r, prod_out);
    return 0;
}

// add_random_number(field2&, min, max, seed) (base/math/random.cpp:24-46): seeded mt19937 uniform noise
// added to the interior cells of an nx x ny row-major field, in place.
int fpref_add_random(int nx, int ny, double lo, double hi, int seed, double* f)
{
    field2 F(nx, ny);
    copy_in(F, f);
    add_random_number(F, lo, hi, seed);
    copy_out(F, f);
    return 0;
}

// The 3D composite: domains[i] = Domain3DUniform(nx, ny, nz, lx, ly, lz) allocated contiguously in index
// order (the address tie-break of TreeUtils::findOptimalRoot then picks the lower index), connect(a, dir, b)
// in order, bc[6 i + face] on every face that is not adjacented (face order x-, x+, y-, y+, z-, z+), one
// Variable3D centre field per domain; ConcatPoissonSolver3D(var) with set_parameter(m, tol, maxIter).
struct Concat3DCase
{
    std::vector<Domain3DUniform>           domains;
    Geometry3D                             geo;
    std::unique_ptr<Variable3D>            var;
    std::vector<field3>                    fields;
    std::unique_ptr<ConcatPoissonSolver3D> solver;
    double                                 t_construct = 0.0;
};

void* fpref_concat3d_create(int nd, const int* nx, const int* ny, const int* nz, const double* lx, const double* ly,
                            const double* lz, int nc, const int* ca, const int* cdir, const int* cb, const int* bc,
                            int m, double tol, int maxIter)
{
    auto* c = new Concat3DCase();
    c->domains.reserve(nd);
    for (int i = 0; i < nd; ++i)
        c->domains.emplace_back(nx[i], ny[i], nz[i], lx[i], ly[i], lz[i], "D" + std::to_string(i));
    for (int i = 0; i < nd; ++i) c->geo.add_domain(&c->domains[i]);
    for (int k = 0; k < nc; ++k) c->geo.connect(&c->domains[ca[k]], loc_of(cdir[k]), &c->domains[cb[k]]);
    c->geo.check();
    c->geo.solve_prepare();
    c->var.reset(new Variable3D("v"));
    c->var->set_geometry(c->geo);
    c->fields.resize(nd);
    for (int i = 0; i < nd; ++i) c->var->set_center_field(&c->domains[i], c->fields[i]);
    for (int i = 0; i < nd; ++i)
        for (int f = 0; f < 6; ++f)
        {
            auto& tm = c->var->boundary_type_map[&c->domains[i]];
            if (tm.count(loc_of(f)) && tm[loc_of(f)] == PDEBoundaryType::Adjacented) continue;
            c->var->set_boundary_type(&c->domains[i], loc_of(f), bc_of(bc[6 * i + f]));
        }
    auto t0 = std::chrono::steady_clock::now();
    c->solver.reset(new ConcatPoissonSolver3D(c->var.get()));
    c->solver->set_parameter(m, tol, maxIter);
    auto t1        = std::chrono::steady_clock::now();
    c->t_construct = std::chrono::duration<double>(t1 - t0).count();
    return c;
}

int fpref_concat3d_tree(void* h, int* root, int* level_of)
{
    auto* c = static_cast<Concat3DCase*>(h);
    for (size_t i = 0; i < c->domains.size(); ++i)
        if (&c->domains[i] == c->geo.tree_root) *root = (int)i;
    for (size_t l = 0; l < c->geo.hierarchical_solve_levels.size(); ++l)
        for (auto* d : c->geo.hierarchical_solve_levels[l]) level_of[d - c->domains.data()] = (int)l;
    return 0;
}

// Fills the fields (value(i, j, k) = rhs[(i ny + j) nz + k]) and the six ghost buffers per domain (x faces
// ny x nz, y faces nx x nz, z faces nx x ny, row-major; NULL = zero), runs solve(), copies the solution out.
double fpref_concat3d_solve(void* h, const double* const* rhs, const double* const* ghosts, double* const* out)
{
    auto*     c  = static_cast<Concat3DCase*>(h);
    const int nd = (int)c->domains.size();
    for (int i = 0; i < nd; ++i)
    {
        field3&      F = c->fields[i];
        const size_t n = (size_t)F.get_nx() * F.get_ny() * F.get_nz();
        std::memcpy(F.value, rhs[i], n * sizeof(double));
        for (int f = 0; f < 6; ++f)
        {
            field2& b = *c->var->buffer_map[&c->domains[i]][loc_of(f)];
            for (int p = 0; p < b.get_nx(); ++p)
                for (int q = 0; q < b.get_ny(); ++q)
                    b(p, q) = (ghosts && ghosts[6 * i + f]) ? ghosts[6 * i + f][(size_t)p * b.get_ny() + q] : 0.0;
        }
    }
    auto t0 = std::chrono::steady_clock::now();
    c->solver->solve();
    auto t1 = std::chrono::steady_clock::now();
    for (int i = 0; i < nd; ++i)
    {
        const field3& F = c->fields[i];
        std::memcpy(out[i], F.value, (size_t)F.get_nx() * F.get_ny() * F.get_nz() * sizeof(double));
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

void fpref_concat3d_destroy(void* h) { delete static_cast<Concat3DCase*>(h); }

}  // extern "C"
