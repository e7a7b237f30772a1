// Host-side 2D field of the drop-in interface: the reference's field2 API and layout
// (base/field/field2.h:6-82): row-major nx x ny doubles, value(i, j) = value[i*ny + j]. Solvers copy
// fields to the GPU and back; nothing here computes on the CPU beyond element access and I/O.
#pragma once

#include "base/location_boundary.h"

#include <string>

class field2
{
public:
    double* value = nullptr;

    field2() {}
    field2(int in_nx, int in_ny);
    field2(int in_nx, int in_ny, const std::string& in_name);
    explicit field2(const std::string& in_name);
    ~field2();
    field2(const field2& rhs);
    field2& operator=(const field2& rhs);
    field2(field2&& rhs) noexcept;
    field2& operator=(field2&& rhs) noexcept;

    void init(int in_nx, int in_ny, const std::string& in_name);
    void init(int in_nx, int in_ny);
    void deinit();

    double& operator()(int i, int j) { return value[(long long)i * ny + j]; }
    double  operator()(int i, int j) const { return value[(long long)i * ny + j]; }

    int               get_nx() const { return nx; }
    int               get_ny() const { return ny; }
    int               get_size_n() const { return size_n; }
    double*           get_ptr(int i, int j) const { return value + (long long)ny * i + j; }
    double*           get_ptr(int i) const { return value + (long long)ny * i; }
    const std::string get_name() const { return name; }
    void              set_name(const std::string& n) { name = n; }
    void              clear(double clear_value = 0.0);
    double            sum() const;
    double            norm() const;
    void              print() const;

    friend void swap(field2& a, field2& b) noexcept;

protected:
    int         nx = 0, ny = 0, size_n = 0;
    std::string name = "Default";
};
