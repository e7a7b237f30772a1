// Host-side infrastructure shared by the C ABI implementation: error reporting, device buffers,
// device-resident transform and rectangle plans.
#pragma once

#include "fp_plan.h"
#include "fp_transform.cuh"

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fpb
{

struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void        set_last_error(const std::string& msg);
const char* last_error();
void        require_device();

// Runs f, converting exceptions to an fp_status code and the thread's last-error message.
template <typename F> int guarded(F&& f)
{
    try
    {
        f();
        set_last_error("");
        return 0;
    }
    catch (const Error& e)
    {
        set_last_error(e.what());
        return e.code;
    }
    catch (const std::exception& e)
    {
        set_last_error(e.what());
        return 1;
    }
    catch (...)
    {
        set_last_error("unknown error");
        return 1;
    }
}

#define FPB_CUDA(call)                                                                                   \
    do                                                                                                   \
    {                                                                                                    \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw ::fpb::Error(e_ == cudaErrorMemoryAllocation ? 6 : 2,                                  \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

// Every kernel launch is followed by FPB_CHECK_LAUNCH(), which also counts it (fp_launch_count()).
void      note_launch();
void      note_launches(long long n);  // kernels of a replayed CUDA graph
long long launches_noted();
#define FPB_CHECK_LAUNCH()                                                                               \
    do                                                                                                   \
    {                                                                                                    \
        ::fpb::note_launch();                                                                            \
        FPB_CUDA(cudaGetLastError());                                                                    \
    } while (0)

// Owning device allocation.
class DevBuf
{
public:
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { alloc(bytes); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&)            = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_)
    {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o)
        {
            release();
            p_   = o.p_;
            n_   = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t bytes)
    {
        release();
        if (bytes == 0) return;
        FPB_CUDA(cudaMalloc(&p_, bytes));
        n_ = bytes;
    }
    void ensure(size_t bytes)
    {
        if (bytes > n_) alloc(bytes);
    }
    void release()
    {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p_); }
    void*  get() const { return p_; }
    size_t bytes() const { return n_; }

private:
    void*  p_ = nullptr;
    size_t n_ = 0;
};

template <typename T> DevBuf upload(const std::vector<T>& v)
{
    DevBuf b(v.size() * sizeof(T));
    if (!v.empty()) FPB_CUDA(cudaMemcpy(b.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return b;
}

// Device-resident plan for one transform family at one row length and precision.
template <typename T> struct DevTransform
{
    typedef typename Cplx<T>::type T2;
    int     kind = 0, n = 0;
    FftDesc fd{}, fd_inv{};  // forward / inverse windows of one plan
    DevBuf  tw, chirp, bhat, bhat_inv, perm, stages, ta, tb, tc;
    XformArgs<T> hargs[2]{};  // args(false), args(true), passed by value to k_b_xform (one plan per launch)
    DevBuf  gscratch;  // eng 2: the FFT buffers of gctas CTAs in global memory, gstride elements each
    T       s1 = 0, s2 = 0;
    int     threads = 128;
    size_t  smem    = 0;
    int     gctas   = 0;
    long long gstride = 0;

    // allow_register false: keep the plan on the stage engine (callers that launch plans of several
    // lengths with one CTA shape). allow_global: rows whose FFT buffer exceeds a CTA's shared memory run
    // with the buffer in global memory (eng 2) instead of being refused (callers that launch this plan
    // alone).
    DevTransform(int kind, int n, bool allow_register = true, bool allow_global = false);
    // Everything but the rows for one direction.
    XformArgs<T> args(bool inverse) const;
    // rows = fields * nx contiguous rows of length n; in and out may alias.
    void run(const T* in, T* out, long long rows, bool inverse, cudaStream_t s) const { run_io<T>(in, out, rows, inverse, s); }
    // Same with rows of another element type (FP64 rows through an FP32 transform).
    template <typename TIO> void run_io(const TIO* in, TIO* out, long long rows, bool inverse, cudaStream_t s) const;
};

// Device-resident PoissonSolver2D: transform plan + chase tables.
template <typename T> struct DevRect
{
    int                              nx = 0, ny = 0;
    double                           hx = 0, hy = 0;
    int                              bc[4]{};
    std::unique_ptr<DevTransform<T>> tr;
    DevBuf                           ctab;  // nx*ny chase coefficients (meaning in fp_chase.cuh)
    DevBuf                           z1, z2;  // periodic-x Sherman-Morrison vectors (nx*ny each)
    bool                             periodic_x = false;
    bool                             singular   = false;  // no Dirichlet-like face: wavenumbers >= sing_from
    int                              sing_from  = 0;      // singular (the last one, ny - 1, except in 3D)
    bool                             chunked    = false;  // partition chase (nx a multiple of kChunk)
    bool                             end_neumann = false;
    DevBuf                           cc, cg, chh, cends, dsep;  // partition chase tables
    DevBuf                           sep_cp, sep_iden;          // separator-system Thomas factors [p][j]
    int                              sep_pmax = 0;              // rows of those tables
    mutable DevBuf                   scratch;                   // partition chase scratch (per batch)

    // sep_rows: separator-factor rows to tabulate (default nx / 32; larger for tables shared by a batch)
    // with_transform false: chase tables only (no transform plan; tr stays null).
    DevRect(int nx, int ny, double hx, double hy, const int* bc, int sep_rows = 0, bool with_transform = true);
    // Chase tables only, for d.size() systems of length nx with diagonals d (the 3D solver's combined
    // z / y modes) and the x boundary types; singular systems are those from sing_from on.
    DevRect(int nx, const std::vector<double>& d, int bc_xneg, int bc_xpos, bool singular, int sing_from);
    void build_chase_tables(const std::vector<double>& d, int sep_rows);
    // In-place solve of `batch` back-to-back fields.
    void solve(T* f, long long batch, cudaStream_t s) const;
    // FP64 plans only: the same solve with FP32 transforms (FP64 rows in and out, FP64 chase); the
    // reduced-precision inner solve of iterative refinement. The FP32 transform plan is built on first use.
    void solve_mixed(T* f, long long batch, cudaStream_t s) const;
    mutable std::unique_ptr<DevTransform<float>> tr32;
    // Scratch elements the partition chase needs for `batch` fields (0 when it is not used).
    long long chase_scratch_elems(long long batch) const;
    // The chase alone, with caller-provided scratch of chase_scratch_elems(batch) elements.
    void chase(T* f, long long batch, T* scratch, cudaStream_t s) const;
    // The chase alone on fields already in transformed space, scratch from the plan.
    void chase_alone(T* f, long long batch, cudaStream_t s) const;
};

constexpr int kMaxDevices = 128;
// Opt-in dynamic shared memory per CTA on the current device (cached per device).
size_t max_dynamic_smem();
// Sets func's MaxDynamicSharedMemorySize to max_dynamic_smem() on the current device, once per device.
// Kernels must have been given that attribute before resident_ctas is asked about them.
void allow_max_dynamic_smem(const void* func);
// CTAs of `threads` threads and `smem` bytes of dynamic shared memory resident on the whole current device.
long long resident_ctas(const void* func, int threads, size_t smem);

}  // namespace fpb

// Handle behind fp_rect* (include/fp_capi.h).
struct fp_rect
{
    int                                    precision = 0;  // FP_F64 or FP_F32
    std::unique_ptr<fpb::DevRect<double>> r64;
    std::unique_ptr<fpb::DevRect<float>>  r32;
    fpb::DevBuf                            staging;
};
