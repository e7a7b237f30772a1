// Host-side plans: FFT factorisation / twiddles, per-boundary-pair transform tables, rectangle
// solver coefficients. Everything here is computed once per plan and uploaded to the device.
#pragma once

#include "fp_fft.cuh"
#include "fp_fft16.cuh"

#include <complex>
#include <string>
#include <vector>

namespace fpb
{

// Boundary types and faces, numbered like the reference's PDEBoundaryType / LocationType
// (base/location_boundary.h:8-16, 62-69).
enum Bc : int
{
    BC_DIRICHLET  = 0,
    BC_NEUMANN    = 1,
    BC_PERIODIC   = 2,
    BC_ADJACENTED = 3,
    BC_NULL       = 4
};
enum Face : int
{
    XNEG = 0,
    XPOS = 1,
    YNEG = 2,
    YPOS = 3
};
inline bool dir_like(int b) { return b == BC_DIRICHLET || b == BC_ADJACENTED; }
inline int  opposite_face(int f) { return f ^ 1; }

// y-transform families, one per boundary pair (PoissonSolver2DBase::create_fft,
// pe/poisson/poisson_solver2d_base.cpp:64-91).
enum Kind : int
{
    K_DD = 0,
    K_NN = 1,
    K_ND = 2,
    K_DN = 3,
    K_PP = 4
};
int kind_of(int bc_neg, int bc_pos);  // -1 if unsupported

// Length of the complex FFT each family's device transform runs (fp_transform.cuh).
int fft_length(int kind, int n);

// Inputs a transform reads and outputs it keeps, for Bluestein's windowed convolution (fp_fft.cuh).
struct FftWindow
{
    int in0, nin, out0, nout;
};
// Window of a family's complex FFT in one direction: the quarter-wave families read elements 1..n and
// keep 1..2n (ND inverse: reads 1..2n, keeps 1..n); the others use the whole length.
FftWindow fft_window(int kind, int n, bool inverse);

struct HostFft
{
    FftDesc                               d{};      // forward window
    FftDesc                               d_inv{};  // inverse window (same M, stages and tables)
    std::vector<std::complex<long double>> tw;     // stage engine: stage twiddles; register engine:
                                                   // exp(-2 pi i m / M), m < M/16
    std::vector<std::complex<long double>> chirp;  // Bluestein: c_n = exp(-i pi n^2 / L), n < L
    std::vector<std::complex<long double>> bhat;      // scaled by 1/M; digit-reversed for the stage engine,
                                                      // natural order for the register engine
    std::vector<std::complex<long double>> bhat_inv;  // kernel of the inverse window, if it differs
    std::vector<int>                       perm;
};
// Plans a length-L complex DFT whose single buffer must fit in smem_limit bytes for complex
// elements of elem_bytes, with the forward and inverse windows fw and iw (used when L needs
// Bluestein): on the register engine (fp_fft16.cuh) when L is a power of two >= 512 or needs Bluestein
// and a power-of-two convolution length fits (and allow_register), else on the stage engine
// (fp_fft.cuh). Throws std::runtime_error if it cannot.
HostFft plan_fft(int L, size_t elem_bytes, size_t smem_limit);
// allow_global: a stage plan whose buffer exceeds smem_limit runs on a buffer in global memory (eng 2)
// instead of being refused.
HostFft plan_fft(int L, size_t elem_bytes, size_t smem_limit, FftWindow fw, FftWindow iw, bool allow_register = true,
                 bool allow_global = false);

// Per-family tables computed with the reference's own double expressions so that the device
// transform reproduces the reference's values, not merely the exact transform.
struct KindTables
{
    std::vector<double> a, b;  // NN: cos/sin(pi (j+1) / n / 2); ND: cos/sin(2 n pi (j+1) / (2n+1));
                               // PP: cos/sin(pi (2j+1) / 4); DD: a = sin(pi j/(n+1)), j <= n (b empty)
    double s1 = 0, s2 = 0;     // DD: sqrt(2/(1+n)); NN: sqrt(2/n), sqrt(1/n); ND/DN: sqrt(4/(2n+1));
                               // PP: sqrt(2/n)
    std::vector<std::complex<long double>> c;  // NN: exp(-i pi m / 2n), m < n
};
KindTables kind_tables(int kind, int n);

// Eigenvalues of the y second difference (PoissonSolver2DBase::cal_lambda,
// pe/poisson/poisson_solver2d_base.cpp:28-62) and the chase diagonal
// x_diag[j] = -2 + hx^2/hy^2 (lambda_j - 2) (pe/poisson/poisson_solver2d.cpp:46-51).
std::vector<double> cal_lambda(int n, int bc_neg, int bc_pos);
std::vector<double> x_diag(int ny, double hx, double hy, int bc_yneg, int bc_ypos);

}  // namespace fpb
