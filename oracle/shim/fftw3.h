/*
 * Oracle-only stand-in for the four FFTW3 symbols the reference's 2D Poisson path uses
 * (pe/poisson/poisson_fft2d.h:6 includes <fftw3.h>; calls at pe/poisson/poisson_fft2d.cpp:34-449).
 *
 * This header is TEST INFRASTRUCTURE. It exists only so that the reference's own serial sources
 * can be compiled into the CPU oracle under oracle/_ref; nothing in the product links it.
 *
 * Semantics restated from FFTW's published definition of the real-to-complex DFT
 * (unnormalised, forward sign):  out[k] = sum_{n=0}^{N-1} in[n] * exp(-2*pi*i*k*n/N),
 * k = 0 .. N/2 (integer division), out[k][0] = real part, out[k][1] = imaginary part.
 * The FFTW3 version the reference was written against is not pinned by the reference
 * (cmake/FindFFTW.cmake; README_en.md:55); any conforming version has these semantics.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];

struct fp_oracle_r2c_plan;
typedef struct fp_oracle_r2c_plan* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
void      fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void      fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
