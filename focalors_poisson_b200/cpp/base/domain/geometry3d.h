// Geometry of boxes of the drop-in interface (reference base/domain/geometry3d.h:14-55): adjacency by face,
// the connectivity check, the tree used by the composite solver (TreeUtils, as in 2D) and axis offsets.
#pragma once

#include "base/domain/domain3d.h"
#include "base/domain/geometry_tree.hpp"
#include "base/location_boundary.h"

#include <unordered_map>
#include <utility>
#include <vector>

class Geometry3D
{
public:
    std::vector<Domain3DUniform*>                                                            domains;
    std::unordered_map<Domain3DUniform*, std::unordered_map<LocationType, Domain3DUniform*>> adjacency;

    bool is_checked  = false;
    bool is_prepared = false;

    Domain3DUniform*                                                                         tree_root = nullptr;
    std::unordered_map<Domain3DUniform*, std::unordered_map<LocationType, Domain3DUniform*>> tree_map;
    std::unordered_map<Domain3DUniform*, std::pair<LocationType, Domain3DUniform*>>          parent_map;
    std::vector<std::vector<Domain3DUniform*>>                                               hierarchical_solve_levels;

    // connect() calls in order (a, direction from a, b): the solver hands them to the device in this order
    std::vector<std::pair<std::pair<Domain3DUniform*, LocationType>, Domain3DUniform*>> connections;

    Geometry3D() = default;
    ~Geometry3D() {}

    void add_domain(Domain3DUniform* s);
    void connect(Domain3DUniform* a, LocationType dir, Domain3DUniform* b);

    void check();
    void solve_prepare();

    void set_global_spatial_step(double hx, double hy, double hz);

    void axis(Domain3DUniform* d, LocationType loc);

    void update_offset_x(Domain3DUniform* d);
    void update_offset_y(Domain3DUniform* d);
    void update_offset_z(Domain3DUniform* d);

    void global_move_x(double x);
    void global_move_y(double y);
    void global_move_z(double z);

    int index_of(const Domain3DUniform* d) const;

private:
    bool is_single_connected() const;
    void build_tree();
};
