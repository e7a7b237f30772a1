// Device-side field set-up (include/fp_capi.h fp_field_fill / fp_buffer_fill): the values
// Variable2D::set_value and Variable2D::set_buffer_value compute on the host
// (base/domain/variable2d.cpp:345-416, 467-511) for analytic right-hand sides given as a sum of separable
// terms, evaluated in one kernel on the device, so that a right-hand side need not be filled on the host
// and copied over.
#include "../../include/fp_capi.h"
#include "fp_internal.h"

namespace fpb
{
namespace
{
constexpr int kMaxTerms = 48;  // 48 terms of 64 bytes: 3 KB of kernel parameters

struct TermSet
{
    int     n;
    fp_term t[kMaxTerms];
};

__device__ __forceinline__ double factor(int kind, const double* p, double x)
{
    switch (kind)
    {
        case FP_FACTOR_SIN: return sin(p[0] * x + p[1]);
        case FP_FACTOR_COS: return cos(p[0] * x + p[1]);
        case FP_FACTOR_GAUSS:
        {
            const double z = (x - p[0]) / p[1];
            return exp(-z * z);
        }
        case FP_FACTOR_QUADRATIC: return p[0] + x * (p[1] + x * p[2]);
        default: return 1.0;
    }
}

__device__ __forceinline__ double eval(const TermSet& ts, double x, double y)
{
    double v = 0.0;
    for (int k = 0; k < ts.n; ++k)
        v += ts.t[k].a * factor(ts.t[k].kind_x, ts.t[k].px, x) * factor(ts.t[k].kind_y, ts.t[k].py, y);
    return v;
}

// f(i, j) (+)= sum of terms at (ox + (i + sx) hx, oy + (j + sy) hy), row-major nx x ny.
__global__ void k_field_fill(double* __restrict__ f, int nx, int ny, double hx, double hy, double ox, double oy,
                             double sx, double sy, const TermSet ts, int accumulate)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * ny) return;
    const int    i = (int)(t / ny), j = (int)(t - (long long)i * ny);
    const double v = eval(ts, ox + (i + sx) * hx, oy + (j + sy) * hy);
    f[t]           = accumulate ? f[t] + v : v;
}

// One ghost buffer: n values at the ghost positions one cell outside `face`.
__global__ void k_buffer_fill(double* __restrict__ b, int n, int face, int nx, int ny, double hx, double hy, double ox,
                              double oy, double sx, double sy, const TermSet ts)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double x, y;
    if (face == 0 || face == 1)
    {
        const int i = face == 0 ? -1 : nx;
        x           = ox + (sx + i) * hx;
        y           = oy + (sy + k) * hy;
    }
    else
    {
        const int j = face == 2 ? -1 : ny;
        x           = ox + (sx + k) * hx;
        y           = oy + (sy + j) * hy;
    }
    b[k] = eval(ts, x, y);
}

// Offsets of value (i, j) from the domain corner in cells, by position (variable2d.cpp:352-370).
void shifts(int position, double& sx, double& sy)
{
    sx = 0.5;
    sy = 0.5;
    switch (position)
    {
        case FP_POS_CENTER: break;
        case FP_POS_XFACE: sx = 0.0; break;
        case FP_POS_YFACE: sy = 0.0; break;
        case FP_POS_CORNER: sx = sy = 0.0; break;
        default: throw Error(FP_ERR_INVALID, "position must be one of FP_POS_*");
    }
}

TermSet terms_of(const fp_term* terms, int nterms)
{
    if (nterms < 0 || nterms > kMaxTerms)
        throw Error(FP_ERR_UNSUPPORTED, "fp_field_fill takes at most " + std::to_string(kMaxTerms) + " terms");
    if (nterms > 0 && !terms) throw Error(FP_ERR_INVALID, "null term list");
    TermSet ts{};
    ts.n = nterms;
    for (int k = 0; k < nterms; ++k)
    {
        ts.t[k] = terms[k];
        for (int kind : {terms[k].kind_x, terms[k].kind_y})
            if (kind < FP_FACTOR_ONE || kind > FP_FACTOR_QUADRATIC) throw Error(FP_ERR_INVALID, "unknown factor kind");
        if ((terms[k].kind_x == FP_FACTOR_GAUSS && terms[k].px[1] == 0.0) ||
            (terms[k].kind_y == FP_FACTOR_GAUSS && terms[k].py[1] == 0.0))
            throw Error(FP_ERR_INVALID, "Gaussian factor of zero width");
    }
    return ts;
}
}  // namespace
}  // namespace fpb

using namespace fpb;

extern "C" {

int fp_field_fill(double* f, int nx, int ny, double hx, double hy, double ox, double oy, int position,
                  const fp_term* terms, int nterms, int accumulate, void* stream)
{
    return guarded([&] {
        if (!f) throw Error(FP_ERR_INVALID, "null field pointer");
        if (nx < 1 || ny < 1) throw Error(FP_ERR_INVALID, "field sizes must be positive");
        double sx, sy;
        shifts(position, sx, sy);
        const TermSet   ts    = terms_of(terms, nterms);
        const long long cells = (long long)nx * ny;
        k_field_fill<<<(unsigned)((cells + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            f, nx, ny, hx, hy, ox, oy, sx, sy, ts, accumulate);
        FPB_CHECK_LAUNCH();
    });
}

int fp_buffer_fill(double* buf, int face, int nx, int ny, double hx, double hy, double ox, double oy, int position,
                   const fp_term* terms, int nterms, void* stream)
{
    return guarded([&] {
        if (!buf) throw Error(FP_ERR_INVALID, "null buffer pointer");
        if (face < 0 || face > 3) throw Error(FP_ERR_INVALID, "face must be 0..3 (LocationType order)");
        if (nx < 1 || ny < 1) throw Error(FP_ERR_INVALID, "field sizes must be positive");
        double sx, sy;
        shifts(position, sx, sy);
        const TermSet ts = terms_of(terms, nterms);
        const int     n  = (face < 2 ? ny : nx) + (position == FP_POS_CORNER ? 1 : 0);
        k_buffer_fill<<<(unsigned)((n + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
            buf, n, face, nx, ny, hx, hy, ox, oy, sx, sy, ts);
        FPB_CHECK_LAUNCH();
    });
}

}  // extern "C"
