// Composite geometry of the drop-in interface (reference base/domain/geometry2d.h:15-59): domains,
// directional adjacency, connectivity check and the domain tree (centre root, BFS levels).
#pragma once

#include "base/location_boundary.h"
#include "domain2d.h"
#include "geometry_tree.hpp"

#include <initializer_list>
#include <stdexcept>
#include <unordered_map>
#include <utility>
#include <vector>

class Geometry2D
{
public:
    std::vector<Domain2DUniform*>                                                            domains;
    std::unordered_map<Domain2DUniform*, std::unordered_map<LocationType, Domain2DUniform*>> adjacency;
    // connect() calls in order: (a, dir, b)
    std::vector<std::pair<std::pair<Domain2DUniform*, LocationType>, Domain2DUniform*>> connections;

    bool is_checked  = false;
    bool is_prepared = false;

    Domain2DUniform*                                                                         tree_root = nullptr;
    std::unordered_map<Domain2DUniform*, std::unordered_map<LocationType, Domain2DUniform*>> tree_map;
    std::unordered_map<Domain2DUniform*, std::pair<LocationType, Domain2DUniform*>>          parent_map;
    std::vector<std::vector<Domain2DUniform*>>                                               hierarchical_solve_levels;

    Geometry2D() = default;
    ~Geometry2D() = default;

    void add_domain(Domain2DUniform* s);
    void add_domain(std::initializer_list<Domain2DUniform*> list);
    void connect(Domain2DUniform* a, LocationType dir, Domain2DUniform* b);

    void check();
    void solve_prepare();

    void set_global_spatial_step(double hx, double hy);
    void axis(Domain2DUniform* d, LocationType loc);
    void update_offset_x(Domain2DUniform* d);
    void update_offset_y(Domain2DUniform* d);
    void global_move_x(double x);
    void global_move_y(double y);

    int index_of(const Domain2DUniform* d) const;

private:
    bool is_single_connected() const;
    void build_tree();
};
