// Uniform box subdomain of the drop-in interface (reference base/domain/domain3d.h:9-86): sizes, lengths, steps
// h = l / n, offsets, the owning geometry and the per-face boundary types.
#pragma once

#include "base/field/field3.h"
#include "base/location_boundary.h"

#include <string>

class Geometry3D;

class Domain3DUniform
{
public:
    int    nx = 0, ny = 0, nz = 0;
    double lx = 0.0, ly = 0.0, lz = 0.0;
    double hx = 0.0, hy = 0.0, hz = 0.0;
    double offset_x = 0.0, offset_y = 0.0, offset_z = 0.0;

    std::string name;
    Geometry3D* parent = nullptr;

    PDEBoundaryType boundary_type_xneg = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_xpos = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_yneg = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_ypos = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_zneg = PDEBoundaryType::Null;
    PDEBoundaryType boundary_type_zpos = PDEBoundaryType::Null;

    Domain3DUniform() = default;
    explicit Domain3DUniform(const std::string& in_name) : name(in_name) {}
    Domain3DUniform(int in_nx, int in_ny, int in_nz, const std::string& in_name)
        : nx(in_nx), ny(in_ny), nz(in_nz), name(in_name)
    {}
    Domain3DUniform(int in_nx, int in_ny, int in_nz, double in_lx, double in_ly, double in_lz,
                    const std::string& in_name)
        : nx(in_nx), ny(in_ny), nz(in_nz), lx(in_lx), ly(in_ly), lz(in_lz), hx(in_lx / in_nx), hy(in_ly / in_ny),
          hz(in_lz / in_nz), name(in_name)
    {}
    ~Domain3DUniform() = default;

    void set_nx(int in_nx)
    {
        nx = in_nx;
        hx = lx / in_nx;
    }
    void set_ny(int in_ny)
    {
        ny = in_ny;
        hy = ly / in_ny;
    }
    void set_nz(int in_nz)
    {
        nz = in_nz;
        hz = lz / in_nz;
    }
    void set_lx(double in_lx)
    {
        lx = in_lx;
        hx = in_lx / nx;
    }
    void set_ly(double in_ly)
    {
        ly = in_ly;
        hy = in_ly / ny;
    }
    void set_lz(double in_lz)
    {
        lz = in_lz;
        hz = in_lz / nz;
    }
    void set_spatial_step(double in_hx, double in_hy, double in_hz)
    {
        hx = in_hx;
        hy = in_hy;
        hz = in_hz;
        lx = nx * hx;
        ly = ny * hy;
        lz = nz * hz;
    }
    void set_size(double in_lx, double in_ly, double in_lz)
    {
        lx = in_lx;
        ly = in_ly;
        lz = in_lz;
        if (nx != 0) hx = in_lx / nx;
        if (ny != 0) hy = in_ly / ny;
        if (nz != 0) hz = in_lz / nz;
    }

    void   set_offset_x(double v) { offset_x = v; }
    void   set_offset_y(double v) { offset_y = v; }
    void   set_offset_z(double v) { offset_z = v; }
    double get_offset_x() const { return offset_x; }
    double get_offset_y() const { return offset_y; }
    double get_offset_z() const { return offset_z; }

    double get_hx() const { return hx; }
    double get_hy() const { return hy; }
    double get_hz() const { return hz; }
    double get_lx() const { return lx; }
    double get_ly() const { return ly; }
    double get_lz() const { return lz; }
    int    get_nx() const { return nx; }
    int    get_ny() const { return ny; }
    int    get_nz() const { return nz; }

    bool check_profile() const { return nx > 0 && ny > 0 && nz > 0 && lx > 0.0 && ly > 0.0 && lz > 0.0; }
    bool check_boundary() const
    {
        return boundary_type_xneg != PDEBoundaryType::Null && boundary_type_xpos != PDEBoundaryType::Null &&
               boundary_type_yneg != PDEBoundaryType::Null && boundary_type_ypos != PDEBoundaryType::Null &&
               boundary_type_zneg != PDEBoundaryType::Null && boundary_type_zpos != PDEBoundaryType::Null;
    }
};
