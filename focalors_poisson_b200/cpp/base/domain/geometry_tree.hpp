// Tree helpers of the drop-in interface (reference base/domain/geometry_tree.hpp:12-250): the tree
// centre by leaf stripping, BFS levels. Geometry2D::build_tree uses them.
#pragma once

#include "base/location_boundary.h"

#include <cstdint>
#include <iostream>
#include <queue>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace TreeUtils
{
template <typename DomainT>
using Adjacency = std::unordered_map<DomainT*, std::unordered_map<LocationType, DomainT*>>;

// Tree centre: strip leaves layer by layer; of two remaining centres the one at the lower address.
template <typename DomainT> DomainT* findOptimalRoot(const Adjacency<DomainT>& adjacency)
{
    if (adjacency.empty()) return nullptr;
    std::unordered_map<DomainT*, int> deg;
    std::vector<DomainT*>             leaves;
    for (const auto& p : adjacency) deg[p.first] = (int)p.second.size();
    for (const auto& p : adjacency)
        if (deg[p.first] <= 1) leaves.push_back(p.first);
    int remaining = (int)adjacency.size();
    while (remaining > 2 && !leaves.empty())
    {
        remaining -= (int)leaves.size();
        std::vector<DomainT*> next;
        for (DomainT* lf : leaves)
            for (const auto& q : adjacency.at(lf))
                if (--deg[q.second] == 1) next.push_back(q.second);
        leaves.swap(next);
    }
    if (leaves.empty()) return adjacency.begin()->first;
    DomainT* root = leaves[0];
    for (DomainT* c : leaves)
        if (reinterpret_cast<uintptr_t>(c) < reinterpret_cast<uintptr_t>(root)) root = c;
    return root;
}

template <typename DomainT>
std::vector<std::vector<DomainT*>> BFS(DomainT* root,
                                       const std::unordered_map<DomainT*, std::unordered_map<LocationType, DomainT*>>& tm)
{
    std::vector<std::vector<DomainT*>> levels;
    if (!root) return levels;
    std::vector<DomainT*> frontier = {root};
    while (!frontier.empty())
    {
        levels.push_back(frontier);
        std::vector<DomainT*> next;
        for (DomainT* d : frontier)
            if (tm.count(d))
                for (const auto& kv : tm.at(d)) next.push_back(kv.second);
        frontier.swap(next);
    }
    return levels;
}

template <typename DomainT>
std::unordered_map<DomainT*, std::unordered_map<LocationType, DomainT*>> buildTreeMapFromRoot(DomainT* root,
                                                                                              const Adjacency<DomainT>& adj)
{
    std::unordered_map<DomainT*, std::unordered_map<LocationType, DomainT*>> tm;
    if (!root) return tm;
    std::vector<std::pair<DomainT*, DomainT*>> stack = {{root, nullptr}};
    std::unordered_set<DomainT*>               seen  = {root};
    while (!stack.empty())
    {
        auto [cur, par] = stack.back();
        stack.pop_back();
        tm.try_emplace(cur);
        if (!adj.count(cur)) continue;
        // children in the adjacency map's own order, as the reference inserts them (the order in which the
        // levels list them)
        for (const auto& kv : adj.at(cur))
        {
            if (kv.second == par) continue;
            if (seen.count(kv.second)) throw std::runtime_error("geometry adjacency has a cycle");
            seen.insert(kv.second);
            tm[cur][kv.first] = kv.second;
            stack.push_back({kv.second, cur});
        }
    }
    return tm;
}

template <typename DomainT>
std::unordered_map<DomainT*, std::pair<LocationType, DomainT*>> buildParentMapFromTree(
    const std::unordered_map<DomainT*, std::unordered_map<LocationType, DomainT*>>& tm)
{
    std::unordered_map<DomainT*, std::pair<LocationType, DomainT*>> pm;
    for (const auto& [d, children] : tm)
        for (const auto& [loc, c] : children) pm[c] = std::make_pair(opposite(loc), d);
    return pm;
}
}  // namespace TreeUtils
