// Variable bound to a composite geometry (reference base/domain/variable2d.h:10-56): one field per
// domain, ghost buffers per face, boundary types.
#pragma once

#include "base/field/field2.h"
#include "domain2d.h"
#include "geometry2d.h"

#include <functional>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <unordered_map>

class Variable2D
{
public:
    std::string                                                                             name;
    Geometry2D*                                                                             geometry = nullptr;
    std::unordered_map<Domain2DUniform*, field2*>                                           field_map;
    std::unordered_map<Domain2DUniform*, std::unordered_map<LocationType, double*>>         buffer_map;
    std::unordered_map<Domain2DUniform*, std::unordered_map<LocationType, PDEBoundaryType>> boundary_type_map;
    VariablePositionType                                                                     position_type =
        VariablePositionType::Null;

    Variable2D() = default;
    explicit Variable2D(const std::string& in_name) : name(in_name) {}
    virtual ~Variable2D();
    Variable2D(const Variable2D&)            = delete;
    Variable2D& operator=(const Variable2D&) = delete;

    virtual void set_geometry(Geometry2D& g);
    virtual void check_geometry(Domain2DUniform* s);
    virtual void set_center_field(Domain2DUniform* s, field2& f);

    virtual void set_boundary_type(Domain2DUniform* s, LocationType loc, PDEBoundaryType type);
    virtual void set_boundary_type(Domain2DUniform* s, std::initializer_list<std::pair<LocationType, PDEBoundaryType>> list);
    virtual void set_boundary_type(PDEBoundaryType type);

    virtual void set_buffer_value(Domain2DUniform* s, LocationType loc, std::function<double(double, double)> f);
    virtual void set_buffer(std::function<double(double, double)> f);
    virtual void set_value(std::function<double(double, double)> func);
};
