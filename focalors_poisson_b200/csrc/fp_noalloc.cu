// fp_rect_solve_f64_noalloc: the rectangle solve for callers that must not allocate device memory at
// solve time: code whose device memory is owned by another allocator (a framework's caching allocator,
// a fixed memory budget), where a library cudaMalloc would either fail or synchronise the device behind
// that allocator's back.
//
// The partition chase of fp_rect_solve_f64 keeps per-call scratch (chunk end values, the separator
// solution and the slopes of the separator scan: 4 * batch * (nx/32) * ny doubles) in a buffer the plan grows with
// cudaMalloc. This variant takes that scratch from one file-scope device array instead, so it calls no
// allocator at all. Limits and sharing rules are stated next to the array below.
#include "../../include/fp_capi.h"
#include "fp_internal.h"

#include <mutex>

namespace
{
// 2^21 doubles = 16 MiB, held on every device that loads this library until the process exits.
constexpr long long kNoallocScratchDoubles = 1LL << 21;
// Shared by every call: it keeps the previous call's contents, and calls whose work overlaps on the
// GPU (different streams, or a second call queued before the first finished on another stream) race on
// it. The chase kernels write every element they later read within one call, so nothing needs clearing.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchDoubles];

// Device address of the array, looked up once per device (with that device current). In host code the
// symbol itself is only a host-side stand-in, never a device address.
double* scratch_address()
{
    static std::mutex mu;
    static double*    addr[fpb::kMaxDevices] = {};
    int               dev                    = 0;
    FPB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= fpb::kMaxDevices) throw fpb::Error(FP_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev])
    {
        void*       p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw fpb::Error(FP_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                                              cudaGetErrorString(e));
        addr[dev] = static_cast<double*>(p);
    }
    return addr[dev];
}
}  // namespace

extern "C" int fp_rect_solve_f64_noalloc(fp_rect* r, double* f, long long batch, void* stream)
{
    return fpb::guarded([&] {
        if (!r || !r->r64) throw fpb::Error(FP_ERR_INVALID, "expected a solver created with FP_F64");
        if (!f) throw fpb::Error(FP_ERR_INVALID, "null field pointer");
        if (batch < 0) throw fpb::Error(FP_ERR_INVALID, "negative batch");
        const fpb::DevRect<double>& plan = *r->r64;
        const long long             need = plan.chase_scratch_elems(batch);
        if (need > kNoallocScratchDoubles)
            throw fpb::Error(FP_ERR_UNSUPPORTED,
                             "fp_rect_solve_f64_noalloc: this solve needs " + std::to_string(need) +
                                 " scratch doubles (4 * batch * (nx/32) * ny); the fixed no-allocation scratch "
                                 "holds " + std::to_string(kNoallocScratchDoubles) + ". Use a smaller batch.");
        double*      scr = scratch_address();
        cudaStream_t s   = static_cast<cudaStream_t>(stream);
        if (batch == 0) return;
        plan.tr->run(f, f, batch * plan.nx, false, s);
        plan.chase(f, batch, scr, s);
        plan.tr->run(f, f, batch * plan.nx, true, s);
    });
}
