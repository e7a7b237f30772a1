// Prints the host-side FFT plan of one transform family and row length (test driver for the CPU test of
// the windowed Bluestein tables): header line, stage radices, chirp, the kernel transforms of the forward
// and inverse windows (scaled by 1/M; digit-reversed on the stage engine, natural order on the register
// engine) and the register engine's rotation table. Third argument: "stage" keeps the plan on the stage
// engine, "register" lets the planner choose. Host code only; no GPU is touched.
#include "../../focalors_poisson_b200/csrc/fp_plan.h"

#include <cstdio>
#include <cstdlib>
#include <string>

using namespace fpb;

static void print_desc(const char* tag, const FftDesc& d)
{
    std::printf("%s %d %d %d %d %d %d %d %d %d\n", tag, d.L, d.M, d.blue, d.in0, d.nin, d.out0, d.nout, d.eng, d.lgM);
}

int main(int argc, char** argv)
{
    if (argc != 4) return 2;
    const int     kind = std::atoi(argv[1]), n = std::atoi(argv[2]);
    const bool    reg  = std::string(argv[3]) == "register";
    const int     L    = fft_length(kind, n);
    const HostFft h = plan_fft(L, 16, (size_t)1 << 30, fft_window(kind, n, false), fft_window(kind, n, true), reg);
    print_desc("fwd", h.d);
    print_desc("inv", h.d_inv);
    std::printf("radices");
    for (int s = 0; s < h.d.nst; ++s) std::printf(" %d", h.d.st[s].R);
    std::printf("\n");
    for (const auto& c : h.chirp) std::printf("c %.21Le %.21Le\n", c.real(), c.imag());
    for (const auto& c : h.bhat) std::printf("b %.21Le %.21Le\n", c.real(), c.imag());
    for (const auto& c : h.bhat_inv) std::printf("i %.21Le %.21Le\n", c.real(), c.imag());
    if (h.d.eng == 1)
        for (const auto& c : h.tw) std::printf("t %.21Le %.21Le\n", c.real(), c.imag());
    return 0;
}
