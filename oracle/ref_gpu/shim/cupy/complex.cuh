// Device stand-in for CuPy's <cupy/complex.cuh> so the reference kernels.cu
// compiles with nvcc (test and baseline infrastructure, oracle/ref_gpu):
// CuPy's complex<T> is a thrust-style complex in the global namespace; the
// libcu++ complex gives the same operations used by kernels.cu (construction
// from (re, im), +, *, abs, real(), imag()).
#pragma once
#include <cuda/std/complex>
template <class T>
using complex = cuda::std::complex<T>;
// abs(z) of a complex argument is found in cuda::std by argument-dependent lookup
