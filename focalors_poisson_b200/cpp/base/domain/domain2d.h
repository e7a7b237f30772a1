// Uniform rectangular subdomain of the drop-in interface (reference base/domain/domain2d.h:10-67).
#pragma once

#include "base/field/field2.h"
#include "base/location_boundary.h"

#include <string>

class Geometry2D;

class Domain2DUniform
{
public:
    int         nx = 0, ny = 0;
    double      lx = 0.0, ly = 0.0;
    double      hx = 0.0, hy = 0.0;
    double      offset_x = 0.0, offset_y = 0.0;
    std::string name;
    Geometry2D* parent = nullptr;

    PDEBoundaryType boundary_type_xneg = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_xpos = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_yneg = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_ypos = PDEBoundaryType::Null;

    Domain2DUniform() = default;
    explicit Domain2DUniform(const std::string& in_name) : name(in_name) {}
    Domain2DUniform(int in_nx, int in_ny, double in_lx, double in_ly, const std::string& in_name)
        : nx(in_nx), ny(in_ny), lx(in_lx), ly(in_ly), hx(in_lx / in_nx), hy(in_ly / in_ny), name(in_name)
    {}
    Domain2DUniform(int in_nx, int in_ny, const std::string& in_name) : nx(in_nx), ny(in_ny), name(in_name) {}

    void set_nx(int v)
    {
        nx = v;
        hx = lx / v;
    }
    void set_ny(int v)
    {
        ny = v;
        hy = ly / v;
    }
    void set_lx(double v)
    {
        lx = v;
        hx = v / nx;
    }
    void set_ly(double v)
    {
        ly = v;
        hy = v / ny;
    }
    void set_spatial_step(double in_hx, double in_hy)
    {
        hx = in_hx;
        hy = in_hy;
        lx = nx * hx;
        ly = ny * hy;
    }
    void set_size(double in_lx, double in_ly)
    {
        lx = in_lx;
        ly = in_ly;
        if (nx != 0) hx = in_lx / nx;
        if (ny != 0) hy = in_ly / ny;
    }
    void   set_offset_x(double v) { offset_x = v; }
    void   set_offset_y(double v) { offset_y = v; }
    double get_offset_x() const { return offset_x; }
    double get_offset_y() const { return offset_y; }
    double get_hx() const { return hx; }
    double get_hy() const { return hy; }
    double get_lx() const { return lx; }
    double get_ly() const { return ly; }
    int    get_nx() const { return nx; }
    int    get_ny() const { return ny; }

    bool check_profile() const { return nx > 0 && ny > 0 && lx > 0.0 && ly > 0.0; }
};
