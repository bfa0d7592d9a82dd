/* Declarations only (test infrastructure, oracle/build_ref.py): the type
 * names src/interp3.cpp's header mentions for AccFFT's plans and complex
 * types; the interpolation kernels use none of them. */
#pragma once
#include <mpi.h>
typedef double Complex[2];
typedef float Complexf[2];
typedef void* fftw_plan;
typedef void* fftwf_plan;
template <typename T, typename Tc, typename Tp>
class accfft_plan_t;
