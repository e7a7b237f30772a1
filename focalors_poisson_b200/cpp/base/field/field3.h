// Host-side 3D field of the drop-in interface: the reference's field3 API and layout
// (base/field/field3.h:8-170): nx x ny x nz doubles, value(i, j, k) = value[(i*ny + j)*nz + k]. Solvers copy
// fields to the GPU and back; the arithmetic here is the host bookkeeping a case file does on fields.
#pragma once

#include "base/field/field2.h"
#include "base/location_boundary.h"

#include <array>
#include <string>

class field3
{
public:
    double* value = nullptr;

    field3() {}
    field3(int in_nx, int in_ny, int in_nz);
    field3(int in_nx, int in_ny, int in_nz, const std::string& in_name);
    explicit field3(const std::string& in_name);
    ~field3();
    field3(const field3& rhs);
    field3& operator=(const field3& rhs);
    field3(field3&& rhs) noexcept { swap(*this, rhs); }
    field3& operator=(field3&& rhs) noexcept
    {
        if (this != &rhs) swap(*this, rhs);
        return *this;
    }

    void init(int in_nx, int in_ny, int in_nz, const std::string& in_name = "");
    void deinit();

    field3  operator+(const field3& rhs);
    field3  operator-(const field3& rhs);
    field3& operator-=(const double a);
    field3  operator*(const double a);
    field3& operator*=(const double a);
    void    add_affine_transform(const double a, const field3& x, const double b);
    void    transpose(field3& dst, const std::array<int, 3>& permutation);

    double norm();
    double sum();
    double sum_at_xy_plane(int k);
    double sum_at_xz_plane(int j);
    double sum_at_yz_plane(int i);
    double squared_sum();
    double mean();
    double mean_at_xy_plane(int k);
    double mean_at_xz_plane(int j);
    double mean_at_yz_plane(int i);

    void xneg_bond_add(const double a, const field2& bound);
    void xpos_bond_add(const double a, const field2& bound);
    void yneg_bond_add(const double a, const field2& bound);
    void back_bond_add(const double a, const field2& bound);
    void zneg_bond_add(const double a, const field2& bound);
    void up_bond_add(const double a, const field2& bound);
    void bond_add(LocationType location, const double a, const field2& bound);

    void xneg_bond_add(const double a, const field3& neighbour);
    void xpos_bond_add(const double a, const field3& neighbour);
    void yneg_bond_add(const double a, const field3& neighbour);
    void back_bond_add(const double a, const field3& neighbour);
    void zneg_bond_add(const double a, const field3& neighbour);
    void up_bond_add(const double a, const field3& neighbour);
    void bond_add(LocationType location, const double a, const field3& neighbour);

    double& operator()(int i, int j, int k) { return value[((long long)i * ny + j) * nz + k]; }
    double  operator()(int i, int j, int k) const { return value[((long long)i * ny + j) * nz + k]; }

    int               get_nx() const { return nx; }
    int               get_ny() const { return ny; }
    int               get_nz() const { return nz; }
    int               get_size_n() const { return size_n; }
    bool              set_size(int in_nx, int in_ny, int in_nz);
    double*           get_ptr(int i, int j, int k) const { return value + ((long long)i * ny + j) * nz + k; }
    const std::string get_name() const { return name; }

    void copy_xz_slice_to(double* dest, int start, int length);
    void copy_xz_slice_from(double* src, int start, int length);
    void copy_xy_block_to(double* dest, int start_x, int start_y, int length_x, int length_y);
    void copy_xy_block_from(double* src, int start_x, int start_y, int length_x, int length_y);

    void clear(double clear_value = 0.0);
    void print() const;

    friend void swap(field3& lhs, field3& rhs) noexcept;

protected:
    int         nx = 0, ny = 0, nz = 0, size_n = 0;
    std::string name = "Default";
};
