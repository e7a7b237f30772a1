// C ABI (include/fp_capi.h): transforms and the single-rectangle solver.
#include "../../include/fp_capi.h"
#include "fp_internal.h"

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

namespace fpb
{
namespace
{
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace
{
std::atomic<long long> g_launches{0};
}
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_noted() { return (long long)g_launches.load(std::memory_order_relaxed); }

const char* last_error() { return g_last_error.c_str(); }

void require_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
    {
        cudaGetLastError();
        throw Error(FP_ERR_CUDA, "no CUDA device available (libfpb200 has no CPU fallback)");
    }
}


namespace
{
// Transform plans cached per (device, family, length, precision).
template <typename T> std::shared_ptr<DevTransform<T>> cached_transform(int kind, int n)
{
    static std::mutex                                                      mu;
    static std::map<std::tuple<int, int, int>, std::shared_ptr<DevTransform<T>>> cache;
    int                                                                    dev = 0;
    FPB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto                        key = std::make_tuple(dev, kind, n);
    auto                        it  = cache.find(key);
    if (it != cache.end()) return it->second;
    auto p     = std::make_shared<DevTransform<T>>(kind, n, true, true);
    cache[key] = p;
    return p;
}

template <typename T>
void transform_impl(int bn, int bp, int nx, int ny, int inverse, const T* in, T* out, int flags, void* stream)
{
    require_device();
    const int kind = kind_of(bn, bp);
    if (kind < 0) throw Error(FP_ERR_INVALID, "unsupported y boundary pair");
    if (nx <= 0) throw Error(FP_ERR_INVALID, "nx must be positive");
    if (!in || !out) throw Error(FP_ERR_INVALID, "null field pointer");
    auto         tr = cached_transform<T>(kind, ny);
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    if (flags & FP_DEVICE)
    {
        tr->run(in, out, nx, inverse != 0, s);
        if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const size_t bytes = (size_t)nx * ny * sizeof(T);
    DevBuf       d(bytes);
    FPB_CUDA(cudaMemcpyAsync(d.get(), in, bytes, cudaMemcpyHostToDevice, s));
    tr->run(d.as<T>(), d.as<T>(), nx, inverse != 0, s);
    FPB_CUDA(cudaMemcpyAsync(out, d.get(), bytes, cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace
}  // namespace fpb

using namespace fpb;


namespace fpb
{
// The whole solve, or with chase_only the chasing step alone (the field is in transformed space).
template <typename T, typename R>
void rect_solve(fp_rect* r, R* plan, T* f, long long batch, int flags, void* stream, bool chase_only = false)
{
    if (!plan) throw Error(FP_ERR_INVALID, "solver was created with the other precision");
    if (!f) throw Error(FP_ERR_INVALID, "null field pointer");
    if (batch < 0) throw Error(FP_ERR_INVALID, "negative batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (flags & FP_DEVICE)
    {
        if (chase_only) plan->chase_alone(f, batch, s);
        else plan->solve(f, batch, s);
        if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const size_t bytes = (size_t)batch * plan->nx * plan->ny * sizeof(T);
    r->staging.ensure(bytes);
    FPB_CUDA(cudaMemcpyAsync(r->staging.get(), f, bytes, cudaMemcpyHostToDevice, s));
    if (chase_only) plan->chase_alone(r->staging.as<T>(), batch, s);
    else plan->solve(r->staging.as<T>(), batch, s);
    FPB_CUDA(cudaMemcpyAsync(f, r->staging.get(), bytes, cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace fpb

extern "C" {

const char* fp_last_error(void) { return fpb::g_last_error.c_str(); }

long long fp_launch_count(void) { return fpb::g_launches.load(); }

int fp_transform_f64(int bn, int bp, int nx, int ny, int inverse, const double* in, double* out, int flags,
                     void* stream)
{
    return guarded([&] { transform_impl<double>(bn, bp, nx, ny, inverse, in, out, flags, stream); });
}

int fp_transform_f32(int bn, int bp, int nx, int ny, int inverse, const float* in, float* out, int flags,
                     void* stream)
{
    return guarded([&] { transform_impl<float>(bn, bp, nx, ny, inverse, in, out, flags, stream); });
}

int fp_rect_create(int nx, int ny, double hx, double hy, const int* bc, int precision, fp_rect** out)
{
    return guarded([&] {
        if (!out || !bc) throw Error(FP_ERR_INVALID, "null argument");
        *out = nullptr;
        require_device();
        std::unique_ptr<fp_rect> r(new fp_rect());
        r->precision = precision;
        if (precision == FP_F64) r->r64.reset(new DevRect<double>(nx, ny, hx, hy, bc));
        else if (precision == FP_F32) r->r32.reset(new DevRect<float>(nx, ny, hx, hy, bc));
        else throw Error(FP_ERR_INVALID, "precision must be FP_F64 or FP_F32");
        *out = r.release();
    });
}


int fp_rect_solve_f64(fp_rect* r, double* f, long long batch, int flags, void* stream)
{
    return guarded([&] {
        if (!r) throw Error(FP_ERR_INVALID, "null solver");
        rect_solve<double>(r, r->r64.get(), f, batch, flags, stream);
    });
}

int fp_rect_solve_f32(fp_rect* r, float* f, long long batch, int flags, void* stream)
{
    return guarded([&] {
        if (!r) throw Error(FP_ERR_INVALID, "null solver");
        rect_solve<float>(r, r->r32.get(), f, batch, flags, stream);
    });
}

int fp_rect_chase_f64(fp_rect* r, double* f, long long batch, int flags, void* stream)
{
    return guarded([&] {
        if (!r) throw Error(FP_ERR_INVALID, "null solver");
        rect_solve<double>(r, r->r64.get(), f, batch, flags, stream, true);
    });
}

int fp_rect_destroy(fp_rect* r)
{
    return guarded([&] { delete r; });
}

}  // extern "C"
