// Boundary and location enums of the drop-in C++ interface, numbered like the reference's
// base/location_boundary.h:8-99 so that case files and the C ABI agree on every value.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <iostream>
#include <stdexcept>

enum class LocationType : std::uint8_t
{
    XNegative,
    XPositive,
    YNegative,
    YPositive,
    ZNegative,
    ZPositive
};

constexpr std::array<LocationType, 4> kBoundaryLocations2D = {LocationType::XNegative, LocationType::XPositive,
                                                              LocationType::YNegative, LocationType::YPositive};
constexpr std::array<LocationType, 6> kBoundaryLocations3D = {LocationType::XNegative, LocationType::XPositive,
                                                              LocationType::YNegative, LocationType::YPositive,
                                                              LocationType::ZNegative, LocationType::ZPositive};

inline LocationType opposite(LocationType l)
{
    switch (l)
    {
        case LocationType::XNegative: return LocationType::XPositive;
        case LocationType::XPositive: return LocationType::XNegative;
        case LocationType::YNegative: return LocationType::YPositive;
        case LocationType::YPositive: return LocationType::YNegative;
        case LocationType::ZNegative: return LocationType::ZPositive;
        case LocationType::ZPositive: return LocationType::ZNegative;
    }
    throw std::invalid_argument("Invalid location type");
}

enum class PDEBoundaryType : std::uint8_t
{
    Dirichlet,
    Neumann,
    Periodic,
    Adjacented,
    Null
};

enum class VariablePositionType : std::uint8_t
{
    Center,
    XFace,
    YFace,
    ZFace,
    Corner,
    Null
};

inline bool isDirLike(PDEBoundaryType t) { return t == PDEBoundaryType::Dirichlet || t == PDEBoundaryType::Adjacented; }

std::ostream& operator<<(std::ostream& os, LocationType type);
std::ostream& operator<<(std::ostream& os, PDEBoundaryType type);
std::ostream& operator<<(std::ostream& os, VariablePositionType type);

namespace std
{
template <> struct hash<LocationType>
{
    std::size_t operator()(const LocationType& k) const { return std::hash<std::uint8_t>()(static_cast<std::uint8_t>(k)); }
};
}  // namespace std
