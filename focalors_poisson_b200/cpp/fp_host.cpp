// Implementation of the drop-in C++ interface (headers under focalors_poisson_b200/cpp/) on top of the
// C ABI of libfpb200 (include/fp_capi.h). Host code only: geometry bookkeeping and field I/O; every solve
// runs on the GPU.
#include "base/config.h"
#include "base/domain/domain2d.h"
#include "base/domain/geometry2d.h"
#include "base/domain/variable2d.h"
#include "base/field/field2.h"
#include "base/location_boundary.h"
#include "pe/concat/concat_solver2d.h"
#include "pe/poisson/poisson_solver2d.h"

#include "fp_capi.h"

#include <algorithm>
#include <cmath>
#include <queue>
#include <unordered_set>
#include <utility>

// ---------------------------------------------------------------------------------------------
// enums
// ---------------------------------------------------------------------------------------------
std::ostream& operator<<(std::ostream& os, LocationType t)
{
    static const char* n[] = {"XNegative", "XPositive", "YNegative", "YPositive", "ZNegative", "ZPositive"};
    return os << ((int)t < 6 ? n[(int)t] : "Unknown");
}
std::ostream& operator<<(std::ostream& os, PDEBoundaryType t)
{
    static const char* n[] = {"Dirichlet", "Neumann", "Periodic", "Adjacented", "Null"};
    return os << ((int)t < 5 ? n[(int)t] : "Unknown");
}
std::ostream& operator<<(std::ostream& os, VariablePositionType t)
{
    static const char* n[] = {"Center", "XFace", "YFace", "ZFace", "Corner", "Null"};
    return os << ((int)t < 6 ? n[(int)t] : "Unknown");
}

// ---------------------------------------------------------------------------------------------
// field2
// ---------------------------------------------------------------------------------------------
field2::field2(int in_nx, int in_ny) { init(in_nx, in_ny); }
field2::field2(int in_nx, int in_ny, const std::string& in_name) { init(in_nx, in_ny, in_name); }
field2::field2(const std::string& in_name) : name(in_name) {}
field2::~field2() { deinit(); }
field2::field2(const field2& rhs) : nx(rhs.nx), ny(rhs.ny), size_n(rhs.size_n), name(rhs.name)
{
    value = size_n ? new double[size_n] : nullptr;
    std::copy(rhs.value, rhs.value + size_n, value);
}
field2& field2::operator=(const field2& rhs)
{
    if (this == &rhs) return *this;
    field2 tmp(rhs);
    swap(*this, tmp);
    return *this;
}
field2::field2(field2&& rhs) noexcept { swap(*this, rhs); }
field2& field2::operator=(field2&& rhs) noexcept
{
    if (this != &rhs) swap(*this, rhs);
    return *this;
}
void field2::init(int in_nx, int in_ny, const std::string& in_name)
{
    init(in_nx, in_ny);
    name = in_name;
}
void field2::init(int in_nx, int in_ny)
{
    if (in_nx < 0 || in_ny < 0) throw std::invalid_argument(name + ": negative field size");
    deinit();
    nx     = in_nx;
    ny     = in_ny;
    size_n = nx * ny;
    value  = new double[size_n];
    clear(0.0);
}
void field2::deinit()
{
    delete[] value;
    value = nullptr;
}
void field2::clear(double v) { std::fill(value, value + size_n, v); }
double field2::sum() const
{
    double s = 0;
    for (int i = 0; i < size_n; ++i) s += value[i];
    return s;
}
double field2::norm() const
{
    double s = 0;
    for (int i = 0; i < size_n; ++i) s += value[i] * value[i];
    return std::sqrt(s);
}
void field2::print() const
{
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) std::cout << (*this)(i, j) << (j == ny - 1 ? '\n' : ',');
}
void swap(field2& a, field2& b) noexcept
{
    std::swap(a.value, b.value);
    std::swap(a.nx, b.nx);
    std::swap(a.ny, b.ny);
    std::swap(a.size_n, b.size_n);
    std::swap(a.name, b.name);
}

// ---------------------------------------------------------------------------------------------
// Geometry2D (reference base/domain/geometry2d.cpp)
// ---------------------------------------------------------------------------------------------
void Geometry2D::add_domain(Domain2DUniform* s)
{
    if (!s) throw std::invalid_argument("add_domain: nullptr");
    if (std::find(domains.begin(), domains.end(), s) == domains.end()) domains.push_back(s);
    s->parent = this;
}
void Geometry2D::add_domain(std::initializer_list<Domain2DUniform*> list)
{
    for (auto* s : list) add_domain(s);
}
void Geometry2D::connect(Domain2DUniform* a, LocationType dir, Domain2DUniform* b)
{
    add_domain({a, b});
    if (dir == LocationType::ZNegative || dir == LocationType::ZPositive)
        throw std::invalid_argument("Geometry2D does not support ZNegative/ZPositive");
    adjacency[a][dir]           = b;
    adjacency[b][opposite(dir)] = a;
    connections.push_back({{a, dir}, b});
    if (dir == LocationType::XNegative || dir == LocationType::XPositive)
    {
        b->set_ly(a->ly);
        b->set_ny(a->ny);
    }
    else
    {
        b->set_lx(a->lx);
        b->set_nx(a->nx);
    }
}
bool Geometry2D::is_single_connected() const
{
    if (domains.empty()) return true;
    if (adjacency.empty()) return domains.size() == 1;
    std::unordered_set<Domain2DUniform*> seen;
    std::queue<Domain2DUniform*>         q;
    q.push(adjacency.begin()->first);
    seen.insert(adjacency.begin()->first);
    while (!q.empty())
    {
        auto* u = q.front();
        q.pop();
        auto it = adjacency.find(u);
        if (it == adjacency.end()) continue;
        for (auto& kv : it->second)
            if (seen.insert(kv.second).second) q.push(kv.second);
    }
    for (auto* s : domains)
        if (!seen.count(s)) return false;
    return true;
}
void Geometry2D::check()
{
    for (auto* s : domains)
        if (!s->check_profile()) throw std::runtime_error("Domain " + s->name + " has invalid profile");
    if (!is_single_connected()) throw std::runtime_error("Geometry is not single connected");
    is_checked = true;
}
void Geometry2D::solve_prepare()
{
    if (!is_checked) throw std::runtime_error("Geometry2D is not checked");
    if (!is_prepared) build_tree();
}
void Geometry2D::build_tree()
{
    tree_root                 = domains.size() == 1 ? domains[0] : TreeUtils::findOptimalRoot(adjacency);
    tree_map                  = TreeUtils::buildTreeMapFromRoot(tree_root, adjacency);
    parent_map                = TreeUtils::buildParentMapFromTree(tree_map);
    hierarchical_solve_levels = TreeUtils::BFS(tree_root, tree_map);
    is_prepared               = true;
}
void Geometry2D::set_global_spatial_step(double hx, double hy)
{
    for (auto* s : domains) s->set_spatial_step(hx, hy);
}
void Geometry2D::axis(Domain2DUniform* d, LocationType loc)
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
        throw std::runtime_error("axis: Invalid LocationType for 2D");
}
void Geometry2D::update_offset_x(Domain2DUniform* d)
{
    std::unordered_set<Domain2DUniform*> seen = {d};
    std::queue<Domain2DUniform*>         q;
    q.push(d);
    while (!q.empty())
    {
        auto* u = q.front();
        q.pop();
        auto it = adjacency.find(u);
        if (it == adjacency.end()) continue;
        for (auto& [dir, v] : it->second)
        {
            if (seen.count(v)) continue;
            double x = u->get_offset_x();
            if (dir == LocationType::XPositive) x += u->get_lx();
            else if (dir == LocationType::XNegative) x -= v->get_lx();
            v->set_offset_x(x);
            seen.insert(v);
            q.push(v);
        }
    }
}
void Geometry2D::update_offset_y(Domain2DUniform* d)
{
    std::unordered_set<Domain2DUniform*> seen = {d};
    std::queue<Domain2DUniform*>         q;
    q.push(d);
    while (!q.empty())
    {
        auto* u = q.front();
        q.pop();
        auto it = adjacency.find(u);
        if (it == adjacency.end()) continue;
        for (auto& [dir, v] : it->second)
        {
            if (seen.count(v)) continue;
            double y = u->get_offset_y();
            if (dir == LocationType::YPositive) y += u->get_ly();
            else if (dir == LocationType::YNegative) y -= v->get_ly();
            v->set_offset_y(y);
            seen.insert(v);
            q.push(v);
        }
    }
}
void Geometry2D::global_move_x(double x)
{
    for (auto* d : domains) d->set_offset_x(d->get_offset_x() + x);
}
void Geometry2D::global_move_y(double y)
{
    for (auto* d : domains) d->set_offset_y(d->get_offset_y() + y);
}
int Geometry2D::index_of(const Domain2DUniform* d) const
{
    auto it = std::find(domains.begin(), domains.end(), d);
    return it == domains.end() ? -1 : (int)(it - domains.begin());
}

// ---------------------------------------------------------------------------------------------
// Variable2D (reference base/domain/variable2d.cpp)
// ---------------------------------------------------------------------------------------------
Variable2D::~Variable2D()
{
    for (auto& kv : buffer_map)
        for (auto& kv2 : kv.second) delete[] kv2.second;
    for (auto& kv : boundary_value_map)
        for (auto& kv2 : kv.second) delete[] kv2.second;
}
void Variable2D::set_geometry(Geometry2D& g)
{
    geometry = &g;
    for (auto& [d, adj] : g.adjacency)
        for (auto& kv : adj) boundary_type_map[d][kv.first] = PDEBoundaryType::Adjacented;
    for (auto* d : g.domains)  // corner node values start at zero for every domain (variable2d.cpp:38-44)
    {
        xneg_ypos_corner_map[d] = 0.0;
        xpos_yneg_corner_map[d] = 0.0;
    }
}
void Variable2D::check_geometry(Domain2DUniform* s)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    if (s->parent != geometry) throw std::runtime_error("Domain not found in geometry");
    if (s->nx <= 0 || s->ny <= 0) throw std::runtime_error("Domain mesh size invalid");
}
// Field of (nx + extra) x (ny + extra) values and four zeroed ghost buffers of the matching lengths
// (reference variable2d.cpp:64-150: extra = 1 for node-centred corner fields, 0 otherwise).
void Variable2D::attach_field(Domain2DUniform* s, field2& f, int extra, VariablePositionType pos)
{
    check_geometry(s);
    f.init(s->nx + extra, s->ny + extra, name + "_" + s->name);
    field_map[s] = &f;
    for (LocationType loc : kBoundaryLocations2D)
    {
        const bool xface = loc == LocationType::XNegative || loc == LocationType::XPositive;
        const int  n     = (xface ? s->ny : s->nx) + extra;
        delete[] buffer_map[s][loc];
        buffer_map[s][loc] = new double[(size_t)n]();
    }
    position_type = pos;
}
void Variable2D::set_center_field(Domain2DUniform* s, field2& f) { attach_field(s, f, 0, VariablePositionType::Center); }
void Variable2D::set_inner_field(Domain2DUniform* s, field2& f) { attach_field(s, f, 0, VariablePositionType::Center); }
void Variable2D::set_x_edge_field(Domain2DUniform* s, field2& f) { attach_field(s, f, 0, VariablePositionType::XFace); }
void Variable2D::set_y_edge_field(Domain2DUniform* s, field2& f) { attach_field(s, f, 0, VariablePositionType::YFace); }
void Variable2D::set_corner_field(Domain2DUniform* s, field2& f) { attach_field(s, f, 1, VariablePositionType::Corner); }

// Offset of value (i, j) from the domain's corner, in cells, for the variable's position
// (variable2d.cpp:231-254): cell centres (0.5, 0.5), x faces (0, 0.5), y faces (0.5, 0), nodes (0, 0).
void Variable2D::position_shift(double& sx, double& sy) const
{
    sx = 0.5;
    sy = 0.5;
    if (position_type == VariablePositionType::XFace) sx = 0.0;
    else if (position_type == VariablePositionType::YFace) sy = 0.0;
    else if (position_type == VariablePositionType::Corner) sx = sy = 0.0;
}
void Variable2D::set_boundary_type(Domain2DUniform* s, LocationType loc, PDEBoundaryType type)
{
    check_geometry(s);
    if (geometry->adjacency.count(s) && geometry->adjacency[s].count(loc))
    {
        if (type != PDEBoundaryType::Adjacented)
            throw std::runtime_error("Attempt to override an adjacented face with non-Adjacented boundary on domain " +
                                     s->name);
        boundary_type_map[s][loc] = PDEBoundaryType::Adjacented;
        return;
    }
    if (boundary_type_map[s].count(loc) && boundary_type_map[s][loc] == PDEBoundaryType::Adjacented &&
        type != PDEBoundaryType::Adjacented)
        throw std::runtime_error("Attempt to change previously Adjacented boundary to another type on domain " +
                                 s->name);
    boundary_type_map[s][loc] = type;
}
void Variable2D::set_boundary_type(Domain2DUniform* s, std::initializer_list<std::pair<LocationType, PDEBoundaryType>> l)
{
    for (const auto& p : l) set_boundary_type(s, p.first, p.second);
}
void Variable2D::set_boundary_type(PDEBoundaryType type)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    for (auto* d : geometry->domains)
        for (LocationType loc : kBoundaryLocations2D)
            if (!boundary_type_map[d].count(loc)) set_boundary_type(d, loc, type);
}
// Constant boundary value on one face (variable2d.cpp:202-224); the x- face value also sets the
// (x-, y+) corner, the y- face value the (x+, y-) corner.
void Variable2D::set_boundary_value(Domain2DUniform* s, LocationType loc, double in_value)
{
    check_geometry(s);
    has_boundary_value_map[s][loc] = true;
    const bool xface = loc == LocationType::XNegative || loc == LocationType::XPositive;
    const int  n     = xface ? s->ny : s->nx;
    double*&   v     = boundary_value_map[s][loc];
    delete[] v;
    v = new double[(size_t)n];
    for (int k = 0; k < n; ++k) v[k] = in_value;
    if (loc == LocationType::XNegative) xneg_ypos_corner_map[s] = in_value;
    if (loc == LocationType::YNegative) xpos_yneg_corner_map[s] = in_value;
}
// Boundary value from f evaluated on the face itself (variable2d.cpp:226-316): the coordinate normal
// to the face is the face's, the tangential one follows the variable's position; node fields have one
// value more along the face.
void Variable2D::set_boundary_value(Domain2DUniform* s, LocationType loc, std::function<double(double, double)> f)
{
    check_geometry(s);
    has_boundary_value_map[s][loc] = true;
    double sx, sy;
    position_shift(sx, sy);
    const bool xface = loc == LocationType::XNegative || loc == LocationType::XPositive;
    const int  extra = position_type == VariablePositionType::Corner ? 1 : 0;
    const int  n     = (xface ? s->ny : s->nx) + extra;
    double*&   v     = boundary_value_map[s][loc];
    delete[] v;
    v = new double[(size_t)n];
    for (int k = 0; k < n; ++k)
    {
        double gx, gy;
        if (xface)
        {
            const int i = loc == LocationType::XNegative ? 0 : s->nx;
            gx          = s->get_offset_x() + i * s->get_hx();
            gy          = s->get_offset_y() + (sy + k) * s->get_hy();
        }
        else
        {
            const int j = loc == LocationType::YNegative ? 0 : s->ny;
            gx          = s->get_offset_x() + (sx + k) * s->get_hx();
            gy          = s->get_offset_y() + j * s->get_hy();
        }
        v[k] = f(gx, gy);
    }
}
// Every non-Adjacented face with a boundary type and no boundary value yet (variable2d.cpp:318-343).
void Variable2D::set_boundary(std::function<double(double, double)> f)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    for (auto& kv : field_map)
    {
        Domain2DUniform* d = kv.first;
        for (LocationType loc : kBoundaryLocations2D)
        {
            auto it = boundary_type_map[d].find(loc);
            if (it == boundary_type_map[d].end() || it->second == PDEBoundaryType::Adjacented ||
                it->second == PDEBoundaryType::Null)
                continue;
            auto hv = has_boundary_value_map[d].find(loc);
            if (hv != has_boundary_value_map[d].end() && hv->second) continue;
            set_boundary_value(d, loc, f);
        }
    }
}
// Ghost buffer of one face: f at the ghost positions one cell outside the face (variable2d.cpp:345-416).
void Variable2D::set_buffer_value(Domain2DUniform* s, LocationType loc, std::function<double(double, double)> f)
{
    check_geometry(s);
    double sx, sy;
    position_shift(sx, sy);
    const bool xface = loc == LocationType::XNegative || loc == LocationType::XPositive;
    const int  extra = position_type == VariablePositionType::Corner ? 1 : 0;
    const int  n     = (xface ? s->ny : s->nx) + extra;
    double*&   buf   = buffer_map[s][loc];
    if (!buf) buf = new double[(size_t)n]();
    for (int k = 0; k < n; ++k)
    {
        double gx, gy;
        if (xface)
        {
            const int i = (loc == LocationType::XNegative) ? -1 : s->nx;
            gx          = s->get_offset_x() + (sx + i) * s->get_hx();
            gy          = s->get_offset_y() + (sy + k) * s->get_hy();
        }
        else
        {
            const int j = (loc == LocationType::YNegative) ? -1 : s->ny;
            gx          = s->get_offset_x() + (sx + k) * s->get_hx();
            gy          = s->get_offset_y() + (sy + j) * s->get_hy();
        }
        buf[k] = f(gx, gy);
    }
}
// Corner node values of staggered fields (variable2d.cpp:418-436): x faces keep the (x+, y-) node
// half a cell below the domain, y faces the (x-, y+) node half a cell left of it.
void Variable2D::set_corner(Domain2DUniform* s, std::function<double(double, double)> f)
{
    check_geometry(s);
    if (position_type == VariablePositionType::XFace)
        xpos_yneg_corner_map[s] = f(s->get_offset_x() + s->nx * s->hx, s->get_offset_y() - 0.5 * s->hy);
    else if (position_type == VariablePositionType::YFace)
        xneg_ypos_corner_map[s] = f(s->get_offset_x() - 0.5 * s->hx, s->get_offset_y() + s->ny * s->hy);
}
void Variable2D::set_buffer(std::function<double(double, double)> f)
{
    if (geometry == nullptr) throw std::runtime_error("Variable2D has no geometry set");
    for (auto& kv : field_map)
        for (LocationType loc : kBoundaryLocations2D)
        {
            auto it = boundary_type_map[kv.first].find(loc);
            if (it == boundary_type_map[kv.first].end() || it->second == PDEBoundaryType::Adjacented ||
                it->second == PDEBoundaryType::Null)
                continue;
            set_buffer_value(kv.first, loc, f);
        }
}
void Variable2D::set_corner(std::function<double(double, double)> f)
{
    for (auto& kv : field_map) set_corner(kv.first, f);
}
void Variable2D::set_value(std::function<double(double, double)> func)
{
    double sx, sy;
    position_shift(sx, sy);
    for (auto& [s, f] : field_map)
        for (int i = 0; i < f->get_nx(); ++i)
            for (int j = 0; j < f->get_ny(); ++j)
                (*f)(i, j) = func(s->get_offset_x() + (sx + i) * s->get_hx(), s->get_offset_y() + (sy + j) * s->get_hy());
}

// ---------------------------------------------------------------------------------------------
// PoissonSolver2D over fp_rect_*
// ---------------------------------------------------------------------------------------------
namespace
{
void fp_check(int rc)
{
    if (rc != FP_OK) throw std::runtime_error(std::string("libfpb200: ") + fp_last_error());
}
}  // namespace

PoissonSolver2D::PoissonSolver2D(int in_nx, int in_ny, double in_hx, double in_hy, PDEBoundaryType bxn,
                                 PDEBoundaryType bxp, PDEBoundaryType byn, PDEBoundaryType byp)
    : nx(in_nx), ny(in_ny)
{
    int bc[4] = {(int)bxn, (int)bxp, (int)byn, (int)byp};
    fp_check(fp_rect_create(nx, ny, in_hx, in_hy, bc, FP_F64, &handle));
}
PoissonSolver2D::PoissonSolver2D(Domain2DUniform* d, Variable2D* v) : nx(d->nx), ny(d->ny)
{
    int bc[4];
    for (int f = 0; f < 4; ++f)
        bc[f] = v ? (int)v->boundary_type_map[d][(LocationType)f] : (int)PDEBoundaryType::Dirichlet;
    fp_check(fp_rect_create(nx, ny, d->hx, d->hy, bc, FP_F64, &handle));
}
PoissonSolver2D::~PoissonSolver2D() { fp_rect_destroy(handle); }
void PoissonSolver2D::solve(field2& f)
{
    if (f.get_nx() != nx || f.get_ny() != ny) throw std::invalid_argument("PoissonSolver2D::solve: field shape mismatch");
    if (EnvironmentConfig::Get().showCurrentStep) std::cout << "[Poisson] solve: start" << std::endl;
    fp_check(fp_rect_solve_f64(handle, f.value, 1, 0, nullptr));
    if (EnvironmentConfig::Get().showCurrentStep) std::cout << "[Poisson] solve: done, f.sum=" << f.sum() << std::endl;
}

// ---------------------------------------------------------------------------------------------
// ConcatPoissonSolver2D over fp_composite_*
// ---------------------------------------------------------------------------------------------
ConcatPoissonSolver2D::ConcatPoissonSolver2D(Variable2D* in_variable) : variable(in_variable) { construct(); }

ConcatPoissonSolver2D::~ConcatPoissonSolver2D()
{
    if (handle) fp_composite_destroy(handle);
}

void ConcatPoissonSolver2D::construct()
{
    if (!variable || !variable->geometry) throw std::runtime_error("ConcatPoissonSolver2D: _variable->geometry is null");
    Geometry2D& g = *variable->geometry;
    if (!g.is_checked) g.check();
    if (g.tree_root == nullptr || g.tree_map.empty()) g.solve_prepare();
    order = g.domains;
    const int           nd = (int)order.size();
    std::vector<int>    nx(nd), ny(nd), bc(4 * nd), conn;
    std::vector<double> hx(nd), hy(nd);
    for (int d = 0; d < nd; ++d)
    {
        Domain2DUniform* s = order[d];
        if (!variable->field_map.count(s)) throw std::runtime_error("ConcatPoissonSolver2D: domain " + s->name + " has no field");
        if (variable->field_map[s]->get_nx() != s->nx || variable->field_map[s]->get_ny() != s->ny)
            throw std::runtime_error("ConcatPoissonSolver2D: field of domain " + s->name +
                                     " is not nx x ny (node-centred corner fields are not solved)");
        nx[d] = s->nx;
        ny[d] = s->ny;
        hx[d] = s->hx;
        hy[d] = s->hy;
        for (int f = 0; f < 4; ++f)
        {
            auto it  = variable->boundary_type_map[s].find((LocationType)f);
            bc[4 * d + f] = it == variable->boundary_type_map[s].end() ? (int)PDEBoundaryType::Null : (int)it->second;
        }
    }
    for (auto& c : g.connections)
    {
        conn.push_back(g.index_of(c.first.first));
        conn.push_back((int)c.first.second);
        conn.push_back(g.index_of(c.second));
    }
    fp_geometry geo{nd, nx.data(), ny.data(), hx.data(), hy.data(), bc.data(), (int)conn.size() / 3,
                    conn.empty() ? nullptr : conn.data(), g.index_of(g.tree_root)};
    if (handle) fp_composite_destroy(handle);
    handle = nullptr;
    fp_check(fp_composite_create(&geo, m, tol, maxIter, 0, &handle));
}

void ConcatPoissonSolver2D::set_parameter(int in_m, double in_tol, int in_maxIter)
{
    const bool changed = (m != in_m) || (tol != in_tol) || (maxIter != in_maxIter);
    m                  = in_m;
    tol                = in_tol;
    maxIter            = in_maxIter;
    if (changed && handle) fp_check(fp_composite_set_parameter(handle, m, tol, maxIter));
}

void ConcatPoissonSolver2D::solve()
{
    if (!handle) throw std::runtime_error("ConcatPoissonSolver2D: not constructed");
    const int                  nd = (int)order.size();
    std::vector<double*>       fields(nd);
    std::vector<const double*> ghosts(4 * nd, nullptr);
    for (int d = 0; d < nd; ++d)
    {
        fields[d] = variable->field_map[order[d]]->value;
        for (int f = 0; f < 4; ++f)
        {
            auto& bm = variable->buffer_map[order[d]];
            auto  it = bm.find((LocationType)f);
            if (it != bm.end()) ghosts[4 * d + f] = it->second;
        }
    }
    fp_solve_info info{};
    fp_check(fp_composite_solve_f64(handle, fields.data(), ghosts.data(), 0, nullptr, &info));
    if (EnvironmentConfig::Get().showGmresRes)
        std::cout << "GMRES: " << info.gmres_iterations << " steps, residual " << info.gmres_residual
                  << (info.converged ? "" : " (not converged)") << std::endl;
}
