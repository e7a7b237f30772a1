// Implementation of the 3D part of the drop-in C++ interface (field3, Geometry3D, Variable3D, PoissonSolver3D,
// ConcatPoissonSolver3D) on top of the C ABI of libfpb200 (include/fp_capi.h). Host code only: geometry
// bookkeeping and field I/O; every solve runs on the GPU.
#include "base/config.h"
#include "base/domain/domain3d.h"
#include "base/domain/geometry3d.h"
#include "base/domain/variable3d.h"
#include "base/field/field2.h"
#include "base/field/field3.h"
#include "base/location_boundary.h"
#include "pe/concat/concat_solver3d.h"
#include "pe/poisson/poisson_solver3d.h"

#include "fp_capi.h"

#include <algorithm>
#include <cmath>
#include <iostream>
#include <queue>
#include <unordered_set>
#include <utility>

// ---------------------------------------------------------------------------------------------
// field3
// ---------------------------------------------------------------------------------------------
field3::field3(int in_nx, int in_ny, int in_nz) { init(in_nx, in_ny, in_nz); }
field3::field3(int in_nx, int in_ny, int in_nz, const std::string& in_name) { init(in_nx, in_ny, in_nz, in_name); }
field3::field3(const std::string& in_name) : name(in_name) {}
field3::~field3() { deinit(); }
field3::field3(const field3& rhs) : nx(rhs.nx), ny(rhs.ny), nz(rhs.nz), size_n(rhs.size_n), name(rhs.name)
{
    value = size_n ? new double[size_n] : nullptr;
    if (size_n) std::copy(rhs.value, rhs.value + size_n, value);
}
// element copy into this field's own extent (both fields are expected to have the same shape)
field3& field3::operator=(const field3& rhs)
{
    if (this != &rhs)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) (*this)(i, j, k) = rhs(i, j, k);
    return *this;
}

void field3::init(int in_nx, int in_ny, int in_nz, const std::string& in_name)
{
    if (in_nx <= 0 || in_ny <= 0 || in_nz <= 0)
        throw std::invalid_argument("field3 " + name + ": sizes must be positive");
    delete[] value;
    nx     = in_nx;
    ny     = in_ny;
    nz     = in_nz;
    name   = in_name;
    size_n = in_nx * in_ny * in_nz;
    value  = new double[size_n]();
}
void field3::deinit()
{
    delete[] value;
    value = nullptr;
}
bool field3::set_size(int in_nx, int in_ny, int in_nz)
{
    if (in_nx * in_ny * in_nz > size_n) return false;
    nx = in_nx;
    ny = in_ny;
    nz = in_nz;
    return true;
}

field3 field3::operator+(const field3& rhs)
{
    field3 r(nx, ny, nz, name);
    for (int t = 0; t < size_n; ++t) r.value[t] = value[t] + rhs.value[t];
    return r;
}
field3 field3::operator-(const field3& rhs)
{
    field3 r(nx, ny, nz, name);
    for (int t = 0; t < size_n; ++t) r.value[t] = value[t] - rhs.value[t];
    return r;
}
field3& field3::operator-=(const double a)
{
    for (int t = 0; t < size_n; ++t) value[t] -= a;
    return *this;
}
field3 field3::operator*(const double a)
{
    field3 r(nx, ny, nz, name);
    for (int t = 0; t < size_n; ++t) r.value[t] = value[t] * a;
    return r;
}
field3& field3::operator*=(const double a)
{
    for (int t = 0; t < size_n; ++t) value[t] *= a;
    return *this;
}
void field3::add_affine_transform(const double a, const field3& x, const double b)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) (*this)(i, j, k) += a * x(i, j, k) + b;
}
void field3::transpose(field3& dst, const std::array<int, 3>& permutation)
{
    const std::array<int, 3> dims = {nx, ny, nz};
    dst.set_size(dims[permutation[0]], dims[permutation[1]], dims[permutation[2]]);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
            {
                const std::array<int, 3> src = {i, j, k};
                dst(src[permutation[0]], src[permutation[1]], src[permutation[2]]) = (*this)(i, j, k);
            }
}

double field3::norm() { return std::sqrt(squared_sum()); }
double field3::sum()
{
    double s = 0.0;
    for (int t = 0; t < size_n; ++t) s += value[t];
    return s;
}
double field3::squared_sum()
{
    double s = 0.0;
    for (int t = 0; t < size_n; ++t) s += value[t] * value[t];
    return s;
}
double field3::mean() { return sum() / (nx * ny * nz); }
double field3::sum_at_xy_plane(int k)
{
    double s = 0.0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) s += (*this)(i, j, k);
    return s;
}
double field3::sum_at_xz_plane(int j)
{
    double s = 0.0;
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) s += (*this)(i, j, k);
    return s;
}
double field3::sum_at_yz_plane(int i)
{
    double s = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) s += (*this)(i, j, k);
    return s;
}
double field3::mean_at_xy_plane(int k) { return sum_at_xy_plane(k) / (nx * ny); }
double field3::mean_at_xz_plane(int j) { return sum_at_xz_plane(j) / (nx * nz); }
double field3::mean_at_yz_plane(int i) { return sum_at_yz_plane(i) / (ny * nz); }

// boundary layers: plane (p, q) of a face, x faces (j, k), y faces (i, k), z faces (i, j)
void field3::xneg_bond_add(const double a, const field2& b)
{
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) (*this)(0, j, k) += a * b(j, k);
}
void field3::xpos_bond_add(const double a, const field2& b)
{
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) (*this)(nx - 1, j, k) += a * b(j, k);
}
void field3::yneg_bond_add(const double a, const field2& b)
{
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) (*this)(i, 0, k) += a * b(i, k);
}
void field3::back_bond_add(const double a, const field2& b)
{
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) (*this)(i, ny - 1, k) += a * b(i, k);
}
void field3::zneg_bond_add(const double a, const field2& b)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) (*this)(i, j, 0) += a * b(i, j);
}
void field3::up_bond_add(const double a, const field2& b)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) (*this)(i, j, nz - 1) += a * b(i, j);
}
void field3::bond_add(LocationType loc, const double a, const field2& b)
{
    switch (loc)
    {
        case LocationType::XNegative: xneg_bond_add(a, b); break;
        case LocationType::XPositive: xpos_bond_add(a, b); break;
        case LocationType::YNegative: yneg_bond_add(a, b); break;
        case LocationType::YPositive: back_bond_add(a, b); break;
        case LocationType::ZNegative: zneg_bond_add(a, b); break;
        case LocationType::ZPositive: up_bond_add(a, b); break;
        default: throw std::invalid_argument("Invalid location type");
    }
}
// the neighbour's layer on the opposite face
void field3::xneg_bond_add(const double a, const field3& n)
{
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) (*this)(0, j, k) += a * n(n.nx - 1, j, k);
}
void field3::xpos_bond_add(const double a, const field3& n)
{
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) (*this)(nx - 1, j, k) += a * n(0, j, k);
}
void field3::yneg_bond_add(const double a, const field3& n)
{
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) (*this)(i, 0, k) += a * n(i, n.ny - 1, k);
}
void field3::back_bond_add(const double a, const field3& n)
{
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) (*this)(i, ny - 1, k) += a * n(i, 0, k);
}
void field3::zneg_bond_add(const double a, const field3& n)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) (*this)(i, j, 0) += a * n(i, j, n.nz - 1);
}
void field3::up_bond_add(const double a, const field3& n)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) (*this)(i, j, nz - 1) += a * n(i, j, 0);
}
void field3::bond_add(LocationType loc, const double a, const field3& n)
{
    switch (loc)
    {
        case LocationType::XNegative: xneg_bond_add(a, n); break;
        case LocationType::XPositive: xpos_bond_add(a, n); break;
        case LocationType::YNegative: yneg_bond_add(a, n); break;
        case LocationType::YPositive: back_bond_add(a, n); break;
        case LocationType::ZNegative: zneg_bond_add(a, n); break;
        case LocationType::ZPositive: up_bond_add(a, n); break;
        default: throw std::invalid_argument("Invalid location type");
    }
}

void field3::copy_xz_slice_to(double* dest, int start, int length)
{
    for (int j = start; j < start + length; ++j)
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k) dest[((long long)(j - start) * nx + i) * nz + k] = (*this)(i, j, k);
}
void field3::copy_xz_slice_from(double* src, int start, int length)
{
    for (int j = start; j < start + length; ++j)
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k) (*this)(i, j, k) = src[((long long)(j - start) * nx + i) * nz + k];
}
void field3::copy_xy_block_to(double* dest, int sx, int sy, int lx, int ly)
{
    for (int i = sx; i < sx + lx; ++i)
        for (int j = sy; j < sy + ly; ++j)
            for (int k = 0; k < nz; ++k) dest[((long long)(i - sx) * ly + (j - sy)) * nz + k] = (*this)(i, j, k);
}
void field3::copy_xy_block_from(double* src, int sx, int sy, int lx, int ly)
{
    for (int i = sx; i < sx + lx; ++i)
        for (int j = sy; j < sy + ly; ++j)
            for (int k = 0; k < nz; ++k) (*this)(i, j, k) = src[((long long)(i - sx) * ly + (j - sy)) * nz + k];
}
void field3::clear(double v) { std::fill(value, value + size_n, v); }
void field3::print() const
{
    for (int i = 0; i < nx; ++i)
    {
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) std::cout << (*this)(i, j, k) << (k == nz - 1 ? '\n' : ',');
        if (i != nx - 1) std::cout << std::endl;
    }
}
void swap(field3& a, field3& b) noexcept
{
    std::swap(a.value, b.value);
    std::swap(a.nx, b.nx);
    std::swap(a.ny, b.ny);
    std::swap(a.nz, b.nz);
    std::swap(a.size_n, b.size_n);
    std::swap(a.name, b.name);
}

// ---------------------------------------------------------------------------------------------
// Geometry3D
// ---------------------------------------------------------------------------------------------
void Geometry3D::add_domain(Domain3DUniform* s)
{
    if (std::find(domains.begin(), domains.end(), s) == domains.end()) domains.push_back(s);
    s->parent = this;
}

// b takes a's cell counts and lengths across the shared face (Geometry3D::connect, geometry3d.cpp:27-60)
void Geometry3D::connect(Domain3DUniform* a, LocationType dir, Domain3DUniform* b)
{
    add_domain(a);
    add_domain(b);
    adjacency[a][dir]           = b;
    adjacency[b][opposite(dir)] = a;
    connections.push_back({{a, dir}, b});
    if (dir == LocationType::XNegative || dir == LocationType::XPositive)
    {
        b->set_ly(a->ly);
        b->set_ny(a->ny);
        b->set_lz(a->lz);
        b->set_nz(a->nz);
    }
    else if (dir == LocationType::YNegative || dir == LocationType::YPositive)
    {
        b->set_lx(a->lx);
        b->set_nx(a->nx);
        b->set_lz(a->lz);
        b->set_nz(a->nz);
    }
    else
    {
        b->set_lx(a->lx);
        b->set_nx(a->nx);
        b->set_ly(a->ly);
        b->set_ny(a->ny);
    }
}

bool Geometry3D::is_single_connected() const
{
    if (domains.empty()) return true;
    if (adjacency.empty()) return domains.size() == 1;
    std::unordered_set<Domain3DUniform*> seen;
    std::queue<Domain3DUniform*>         q;
    q.push(adjacency.begin()->first);
    seen.insert(adjacency.begin()->first);
    while (!q.empty())
    {
        Domain3DUniform* u = q.front();
        q.pop();
        auto it = adjacency.find(u);
        if (it == adjacency.end()) continue;
        for (const auto& kv : it->second)
            if (kv.second && !seen.count(kv.second))
            {
                seen.insert(kv.second);
                q.push(kv.second);
            }
    }
    for (auto* s : domains)
        if (!seen.count(s)) return false;
    return true;
}

void Geometry3D::check()
{
    for (auto* s : domains)
        if (!s->check_profile()) throw std::runtime_error("Domain " + s->name + " has invalid profile");
    if (!is_single_connected()) throw std::runtime_error("Geometry is not single connected");
    is_checked = true;
}

void Geometry3D::solve_prepare()
{
    if (!is_checked) throw std::runtime_error("Geometry3D is not checked");
    if (!is_prepared) build_tree();
}

void Geometry3D::build_tree()
{
    tree_root                 = domains.size() == 1 ? domains[0] : TreeUtils::findOptimalRoot(adjacency);
    tree_map                  = TreeUtils::buildTreeMapFromRoot(tree_root, adjacency);
    parent_map                = TreeUtils::buildParentMapFromTree(tree_map);
    hierarchical_solve_levels = TreeUtils::BFS(tree_root, tree_map);
    is_prepared               = true;
}

void Geometry3D::set_global_spatial_step(double hx, double hy, double hz)
{
    for (auto* s : domains) s->set_spatial_step(hx, hy, hz);
}

// offsets along the axis of `loc` with d's face `loc` at 0, propagated breadth-first through the adjacency
void Geometry3D::axis(Domain3DUniform* d, LocationType loc)
{
    if (std::find(domains.begin(), domains.end(), d) == domains.end())
        throw std::runtime_error("axis: Domain is not in geometry");
    if (loc == LocationType::XNegative || loc == LocationType::XPositive)
    {
        d->set_offset_x(loc == LocationType::XNegative ? 0.0 : -d->get_lx());
        update_offset_x(d);
    }
    else if (loc == LocationType::YNegative || loc == LocationType::YPositive)
    {
        d->set_offset_y(loc == LocationType::YNegative ? 0.0 : -d->get_ly());
        update_offset_y(d);
    }
    else
    {
        d->set_offset_z(loc == LocationType::ZNegative ? 0.0 : -d->get_lz());
        update_offset_z(d);
    }
}

namespace
{
// Breadth-first from d: a neighbour across the axis' positive face starts where u ends, one across the negative
// face ends where u starts, any other neighbour shares u's offset.
template <typename Get, typename Set, typename Len>
void propagate(std::unordered_map<Domain3DUniform*, std::unordered_map<LocationType, Domain3DUniform*>>& adj,
               Domain3DUniform* d, LocationType neg, LocationType pos, Get get, Set set, Len len)
{
    std::unordered_set<Domain3DUniform*> seen{d};
    std::queue<Domain3DUniform*>         q;
    q.push(d);
    while (!q.empty())
    {
        Domain3DUniform* u = q.front();
        q.pop();
        auto it = adj.find(u);
        if (it == adj.end()) continue;
        for (const auto& kv : it->second)
        {
            Domain3DUniform* v = kv.second;
            if (seen.count(v)) continue;
            double o = get(u);
            if (kv.first == pos) o = get(u) + len(u);
            else if (kv.first == neg) o = get(u) - len(v);
            set(v, o);
            seen.insert(v);
            q.push(v);
        }
    }
}
}  // namespace

void Geometry3D::update_offset_x(Domain3DUniform* d)
{
    propagate(adjacency, d, LocationType::XNegative, LocationType::XPositive,
              [](Domain3DUniform* s) { return s->get_offset_x(); },
              [](Domain3DUniform* s, double v) { s->set_offset_x(v); }, [](Domain3DUniform* s) { return s->get_lx(); });
}
void Geometry3D::update_offset_y(Domain3DUniform* d)
{
    propagate(adjacency, d, LocationType::YNegative, LocationType::YPositive,
              [](Domain3DUniform* s) { return s->get_offset_y(); },
              [](Domain3DUniform* s, double v) { s->set_offset_y(v); }, [](Domain3DUniform* s) { return s->get_ly(); });
}
void Geometry3D::update_offset_z(Domain3DUniform* d)
{
    propagate(adjacency, d, LocationType::ZNegative, LocationType::ZPositive,
              [](Domain3DUniform* s) { return s->get_offset_z(); },
              [](Domain3DUniform* s, double v) { s->set_offset_z(v); }, [](Domain3DUniform* s) { return s->get_lz(); });
}
void Geometry3D::global_move_x(double x)
{
    for (auto* d : domains) d->set_offset_x(d->get_offset_x() + x);
}
void Geometry3D::global_move_y(double y)
{
    for (auto* d : domains) d->set_offset_y(d->get_offset_y() + y);
}
void Geometry3D::global_move_z(double z)
{
    for (auto* d : domains) d->set_offset_z(d->get_offset_z() + z);
}
int Geometry3D::index_of(const Domain3DUniform* d) const
{
    for (size_t i = 0; i < domains.size(); ++i)
        if (domains[i] == d) return (int)i;
    throw std::runtime_error("Domain not found in geometry");
}

// ---------------------------------------------------------------------------------------------
// Variable3D
// ---------------------------------------------------------------------------------------------
Variable3D::~Variable3D()
{
    for (auto& d : boundary_value_map)
        for (auto& l : d.second) delete l.second;
    for (auto& d : buffer_map)
        for (auto& l : d.second) delete l.second;
    for (auto* m : {&corner_x_map, &corner_y_map, &corner_z_map})
        for (auto& p : *m) delete[] p.second;
}

void Variable3D::set_geometry(Geometry3D& g)
{
    geometry = &g;
    for (auto& da : geometry->adjacency)
        for (auto& ln : da.second) boundary_type_map[da.first][ln.first] = PDEBoundaryType::Adjacented;
}

void Variable3D::check_geometry(Domain3DUniform* s)
{
    if (geometry == nullptr) throw std::runtime_error("Variable3D has no geometry set");
    if (s->parent != geometry) throw std::runtime_error("Domain not found in geometry");
    if (s->nx <= 0 || s->ny <= 0 || s->nz <= 0) throw std::runtime_error("Domain mesh size invalid");
}

// A field of nx x ny x nz values at `pos` and a ghost plane per face; the face-centred positions also keep the
// values along two edges (corner maps), as the reference allocates them.
void Variable3D::attach_field(Domain3DUniform* s, field3& f, VariablePositionType pos)
{
    check_geometry(s);
    f.init(s->nx, s->ny, s->nz, name + "_" + s->name);
    field_map[s] = &f;
    auto& b      = buffer_map[s];
    for (auto& l : b) delete l.second;
    b[LocationType::XNegative] = new field2(s->ny, s->nz);
    b[LocationType::XPositive] = new field2(s->ny, s->nz);
    b[LocationType::YNegative] = new field2(s->nx, s->nz);
    b[LocationType::YPositive] = new field2(s->nx, s->nz);
    b[LocationType::ZNegative] = new field2(s->nx, s->ny);
    b[LocationType::ZPositive] = new field2(s->nx, s->ny);
    auto edge = [](std::unordered_map<Domain3DUniform*, double*>& m, Domain3DUniform* d, int n) {
        delete[] m[d];
        m[d] = new double[(size_t)n]();
    };
    if (pos == VariablePositionType::XFace)
    {
        edge(corner_y_map, s, s->ny);
        edge(corner_z_map, s, s->nz);
    }
    else if (pos == VariablePositionType::YFace)
    {
        edge(corner_x_map, s, s->nx);
        edge(corner_z_map, s, s->nz);
    }
    else if (pos == VariablePositionType::ZFace)
    {
        edge(corner_x_map, s, s->nx);
        edge(corner_y_map, s, s->ny);
    }
    position_type = pos;
}

void Variable3D::set_center_field(Domain3DUniform* s, field3& f) { attach_field(s, f, VariablePositionType::Center); }
void Variable3D::set_x_face_center_field(Domain3DUniform* s, field3& f) { attach_field(s, f, VariablePositionType::XFace); }
void Variable3D::set_y_face_center_field(Domain3DUniform* s, field3& f) { attach_field(s, f, VariablePositionType::YFace); }
void Variable3D::set_z_face_center_field(Domain3DUniform* s, field3& f) { attach_field(s, f, VariablePositionType::ZFace); }

// offsets of value (i, j, k) from the box corner in cells, by position (variable3d.cpp:450-478)
void Variable3D::position_shift(double& sx, double& sy, double& sz) const
{
    sx = sy = sz = 0.5;
    switch (position_type)
    {
        case VariablePositionType::XFace: sx = 0.0; break;
        case VariablePositionType::YFace: sy = 0.0; break;
        case VariablePositionType::ZFace: sz = 0.0; break;
        case VariablePositionType::Corner: sx = sy = sz = 0.0; break;
        default: break;
    }
}

void Variable3D::set_boundary_type(Domain3DUniform* s, LocationType loc, PDEBoundaryType type)
{
    check_geometry(s);
    if (geometry && geometry->adjacency.count(s) && geometry->adjacency[s].count(loc))
    {
        if (type != PDEBoundaryType::Adjacented)
            throw std::runtime_error("Attempt to override an adjacented face with non-Adjacented boundary on domain " +
                                     s->name);
        boundary_type_map[s][loc] = PDEBoundaryType::Adjacented;
        return;
    }
    if (boundary_type_map[s].count(loc) && boundary_type_map[s][loc] == PDEBoundaryType::Adjacented &&
        type != PDEBoundaryType::Adjacented)
        throw std::runtime_error("Attempt to change previously Adjacented boundary to another type on domain " + s->name);
    boundary_type_map[s][loc] = type;
}
void Variable3D::set_boundary_type(Domain3DUniform* s, std::initializer_list<std::pair<LocationType, PDEBoundaryType>> l)
{
    for (const auto& p : l) set_boundary_type(s, p.first, p.second);
}
void Variable3D::set_boundary_type(PDEBoundaryType type)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    static const LocationType all[6] = {LocationType::XNegative, LocationType::XPositive, LocationType::YNegative,
                                        LocationType::YPositive, LocationType::ZNegative, LocationType::ZPositive};
    for (auto* d : geometry->domains)
    {
        auto& tm = boundary_type_map[d];
        for (LocationType loc : all)
            if (tm.find(loc) == tm.end()) set_boundary_type(d, loc, type);
    }
}

namespace
{
// The plane of `loc` on box s: its extent (np x nq, one more per side at the Corner position), the fixed cell
// index `fixed` along the face's axis, and a function evaluated at each plane cell with the shifts sx, sy, sz.
template <typename F>
void fill_plane(field2& out, const Domain3DUniform* s, LocationType loc, bool corner, int fixed, double sx, double sy,
                double sz, F&& f)
{
    const int c  = corner ? 1 : 0;
    const int ax = (int)loc >> 1;
    const int np = ax == 0 ? s->ny + c : s->nx + c;
    const int nq = ax == 2 ? s->ny + c : s->nz + c;
    for (int p = 0; p < np; ++p)
        for (int q = 0; q < nq; ++q)
        {
            const int    i = ax == 0 ? fixed : p, j = ax == 0 ? p : (ax == 1 ? fixed : q), k = ax == 2 ? fixed : q;
            const double x = s->get_offset_x() + (sx + i) * s->get_hx();
            const double y = s->get_offset_y() + (sy + j) * s->get_hy();
            const double z = s->get_offset_z() + (sz + k) * s->get_hz();
            out(p, q)      = f(x, y, z);
        }
}
}  // namespace

void Variable3D::set_boundary_value(Domain3DUniform* s, LocationType loc, double in_value)
{
    check_geometry(s);
    has_boundary_value_map[s][loc] = true;
    const int ax                   = (int)loc >> 1;
    delete boundary_value_map[s][loc];
    boundary_value_map[s][loc] = ax == 0 ? new field2(s->ny, s->nz) : (ax == 1 ? new field2(s->nx, s->nz) : new field2(s->nx, s->ny));
    boundary_value_map[s][loc]->clear(in_value);
}

// values on the boundary face itself (the face's axis shift is 0, index 0 or n), variable3d.cpp:265-412
void Variable3D::set_boundary_value(Domain3DUniform* s, LocationType loc, std::function<double(double, double, double)> f)
{
    check_geometry(s);
    has_boundary_value_map[s][loc] = true;
    double sx, sy, sz;
    position_shift(sx, sy, sz);
    const int  ax     = (int)loc >> 1;
    const bool corner = position_type == VariablePositionType::Corner;
    const int  c      = corner ? 1 : 0;
    (ax == 0 ? sx : (ax == 1 ? sy : sz)) = 0.0;
    const bool hi    = ((int)loc & 1) != 0;
    const int  fixed = hi ? (ax == 0 ? s->nx : (ax == 1 ? s->ny : s->nz)) : 0;
    delete boundary_value_map[s][loc];
    boundary_value_map[s][loc] = ax == 0 ? new field2(s->ny + c, s->nz + c)
                                         : (ax == 1 ? new field2(s->nx + c, s->nz + c) : new field2(s->nx + c, s->ny + c));
    fill_plane(*boundary_value_map[s][loc], s, loc, corner, fixed, sx, sy, sz, f);
}

void Variable3D::set_boundary(std::function<double(double, double, double)> f)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    static const LocationType all[6] = {LocationType::XNegative, LocationType::XPositive, LocationType::YNegative,
                                        LocationType::YPositive, LocationType::ZNegative, LocationType::ZPositive};
    for (auto kv : field_map)
    {
        Domain3DUniform* d  = kv.first;
        auto&            tm = boundary_type_map[d];
        auto&            hm = has_boundary_value_map[d];
        for (LocationType loc : all)
        {
            auto t = tm.find(loc);
            if (t == tm.end() || t->second == PDEBoundaryType::Adjacented || t->second == PDEBoundaryType::Null) continue;
            auto h = hm.find(loc);
            if (h != hm.end() && h->second) continue;
            set_boundary_value(d, loc, f);
        }
    }
}

// ghost values one cell outside the face (index -1 or n along its axis), variable3d.cpp:441-561
void Variable3D::set_buffer_value(Domain3DUniform* s, LocationType loc, std::function<double(double, double, double)> f)
{
    check_geometry(s);
    double sx, sy, sz;
    position_shift(sx, sy, sz);
    const int  ax    = (int)loc >> 1;
    const bool hi    = ((int)loc & 1) != 0;
    const int  fixed = hi ? (ax == 0 ? s->nx : (ax == 1 ? s->ny : s->nz)) : -1;
    // the ghost planes are allocated n-by-n (no position of this class carries n + 1 values per side)
    fill_plane(*buffer_map[s][loc], s, loc, false, fixed, sx, sy, sz, f);
}

void Variable3D::set_buffer(std::function<double(double, double, double)> f)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    static const LocationType all[6] = {LocationType::XNegative, LocationType::XPositive, LocationType::YNegative,
                                        LocationType::YPositive, LocationType::ZNegative, LocationType::ZPositive};
    for (auto kv : field_map)
    {
        auto& tm = boundary_type_map[kv.first];
        for (LocationType loc : all)
        {
            auto t = tm.find(loc);
            if (t == tm.end() || t->second == PDEBoundaryType::Adjacented || t->second == PDEBoundaryType::Null) continue;
            set_buffer_value(kv.first, loc, f);
        }
    }
}

// values along two edges of the box for the face-centred positions, with the reference's coordinates
// (variable3d.cpp:563-612: the coordinate along the edge is taken from the box's own origin)
void Variable3D::set_corner(Domain3DUniform* s, std::function<double(double, double, double)> f)
{
    check_geometry(s);
    if (position_type == VariablePositionType::XFace)
    {
        const double x = s->get_offset_x() + s->nx * s->hx;
        for (int j = 0; j < s->ny; j++) corner_y_map[s][j] = f(x, (j + 0.5) * s->hy, s->get_offset_z() - 0.5 * s->hz);
        for (int k = 0; k < s->nz; k++) corner_z_map[s][k] = f(x, s->get_offset_y() - 0.5 * s->hy, (k + 0.5) * s->hz);
    }
    else if (position_type == VariablePositionType::YFace)
    {
        const double y = s->get_offset_y() + s->ny * s->hy;
        for (int i = 0; i < s->nx; i++) corner_x_map[s][i] = f((i + 0.5) * s->hx, y, s->get_offset_z() - 0.5 * s->hz);
        for (int k = 0; k < s->nz; k++) corner_z_map[s][k] = f(s->get_offset_x() - 0.5 * s->hx, y, (k + 0.5) * s->hz);
    }
    else if (position_type == VariablePositionType::ZFace)
    {
        const double z = s->get_offset_z() + s->nz * s->hz;
        for (int i = 0; i < s->nx; i++) corner_x_map[s][i] = f((i + 0.5) * s->hx, s->get_offset_y() - 0.5 * s->hy, z);
        for (int j = 0; j < s->ny; j++) corner_y_map[s][j] = f(s->get_offset_x() - 0.5 * s->hx, (j + 0.5) * s->hy, z);
    }
}
void Variable3D::set_corner(std::function<double(double, double, double)> f)
{
    for (auto kv : field_map) set_corner(kv.first, f);
}

void Variable3D::set_value(std::function<double(double, double, double)> func)
{
    double sx, sy, sz;
    position_shift(sx, sy, sz);
    for (auto& p : field_map)
    {
        Domain3DUniform* s = p.first;
        field3&          f = *p.second;
        for (int i = 0; i < f.get_nx(); ++i)
            for (int j = 0; j < f.get_ny(); ++j)
                for (int k = 0; k < f.get_nz(); ++k)
                    f(i, j, k) = func(s->get_offset_x() + (sx + i) * s->get_hx(), s->get_offset_y() + (sy + j) * s->get_hy(),
                                      s->get_offset_z() + (sz + k) * s->get_hz());
    }
}

// ---------------------------------------------------------------------------------------------
// PoissonSolver3D over fp_rect3d_*, ConcatPoissonSolver3D over fp_composite3d_*
// ---------------------------------------------------------------------------------------------
namespace
{
void fp_check3(int rc)
{
    if (rc != FP_OK) throw std::runtime_error(std::string("libfpb200: ") + fp_last_error());
}
}  // namespace

PoissonSolver3D::PoissonSolver3D(int in_nx, int in_ny, int in_nz, double in_hx, double in_hy, double in_hz,
                                 PDEBoundaryType bxn, PDEBoundaryType bxp, PDEBoundaryType byn, PDEBoundaryType byp,
                                 PDEBoundaryType bzn, PDEBoundaryType bzp)
    : nx(in_nx), ny(in_ny), nz(in_nz)
{
    int bc[6] = {(int)bxn, (int)bxp, (int)byn, (int)byp, (int)bzn, (int)bzp};
    fp_check3(fp_rect3d_create(nx, ny, nz, in_hx, in_hy, in_hz, bc, &handle));
}
PoissonSolver3D::PoissonSolver3D(Domain3DUniform* d, Variable3D* v) : nx(d->nx), ny(d->ny), nz(d->nz)
{
    int bc[6];
    for (int f = 0; f < 6; ++f)
        bc[f] = v ? (int)v->boundary_type_map[d][(LocationType)f] : (int)PDEBoundaryType::Dirichlet;
    fp_check3(fp_rect3d_create(nx, ny, nz, d->hx, d->hy, d->hz, bc, &handle));
}
PoissonSolver3D::~PoissonSolver3D() { fp_rect3d_destroy(handle); }
void PoissonSolver3D::solve(field3& f)
{
    if (f.get_nx() != nx || f.get_ny() != ny || f.get_nz() != nz)
        throw std::invalid_argument("PoissonSolver3D::solve: field shape mismatch");
    fp_check3(fp_rect3d_solve_f64(handle, f.value, 1, 0, nullptr));
}

ConcatPoissonSolver3D::ConcatPoissonSolver3D(Variable3D* in_variable) : variable(in_variable) { construct(); }
ConcatPoissonSolver3D::~ConcatPoissonSolver3D()
{
    if (handle) fp_composite3d_destroy(handle);
}

// init_before_constructing_solver + construct_solver_map (concat_solver3d.cpp:20-98): the geometry is checked
// and its tree built, the boxes, boundary types and connect() calls go to the device solver, which builds the
// Schur matrices
void ConcatPoissonSolver3D::construct()
{
    if (!variable || !variable->geometry) throw std::runtime_error("ConcatPoissonSolver3D: _variable->geometry is null");
    Geometry3D& g = *variable->geometry;
    if (!g.is_checked) g.check();
    if (g.tree_root == nullptr || g.tree_map.empty()) g.solve_prepare();
    order                    = g.domains;
    const int           nd   = (int)order.size();
    std::vector<int>    n[3] = {std::vector<int>(nd), std::vector<int>(nd), std::vector<int>(nd)};
    std::vector<double> h[3] = {std::vector<double>(nd), std::vector<double>(nd), std::vector<double>(nd)};
    std::vector<int>    bc(6 * nd), conn;
    for (int d = 0; d < nd; ++d)
    {
        Domain3DUniform* s = order[d];
        if (!variable->field_map.count(s)) throw std::runtime_error("ConcatPoissonSolver3D: domain " + s->name + " has no field");
        n[0][d] = s->nx;
        n[1][d] = s->ny;
        n[2][d] = s->nz;
        h[0][d] = s->hx;
        h[1][d] = s->hy;
        h[2][d] = s->hz;
        for (int f = 0; f < 6; ++f)
        {
            auto it        = variable->boundary_type_map[s].find((LocationType)f);
            bc[6 * d + f] = it == variable->boundary_type_map[s].end() ? (int)PDEBoundaryType::Null : (int)it->second;
        }
    }
    for (auto& c : g.connections)
    {
        conn.push_back(g.index_of(c.first.first));
        conn.push_back((int)c.first.second);
        conn.push_back(g.index_of(c.second));
    }
    fp_geometry3 geo{nd,          n[0].data(), n[1].data(), n[2].data(), h[0].data(), h[1].data(), h[2].data(),
                     bc.data(),   (int)conn.size() / 3,     conn.empty() ? nullptr : conn.data(),  g.index_of(g.tree_root)};
    if (handle) fp_composite3d_destroy(handle);
    handle = nullptr;
    fp_check3(fp_composite3d_create(&geo, m, tol, maxIter, &handle));
}

void ConcatPoissonSolver3D::set_parameter(int in_m, double in_tol, int in_maxIter)
{
    const bool changed = (m != in_m) || (tol != in_tol) || (maxIter != in_maxIter);
    m                  = in_m;
    tol                = in_tol;
    maxIter            = in_maxIter;
    if (changed && handle) fp_check3(fp_composite3d_set_parameter(handle, m, tol, maxIter));
}

void ConcatPoissonSolver3D::solve()
{
    if (!handle) throw std::runtime_error("ConcatPoissonSolver3D: not constructed");
    const int                  nd = (int)order.size();
    std::vector<double*>       fields(nd);
    std::vector<const double*> ghosts(6 * nd, nullptr);
    for (int d = 0; d < nd; ++d)
    {
        fields[d] = variable->field_map[order[d]]->value;
        auto& bm  = variable->buffer_map[order[d]];
        for (int f = 0; f < 6; ++f)
        {
            auto it = bm.find((LocationType)f);
            if (it != bm.end()) ghosts[6 * d + f] = it->second->value;
        }
    }
    fp_solve_info info{};
    fp_check3(fp_composite3d_solve_f64(handle, fields.data(), ghosts.data(), 0, nullptr, &info));
    if (EnvironmentConfig::Get().showGmresRes)
        std::cout << "GMRES3D: " << info.gmres_iterations << " steps, residual " << info.gmres_residual
                  << (info.converged ? "" : " (not converged)") << std::endl;
}
