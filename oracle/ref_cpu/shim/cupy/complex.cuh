// Host stand-in for CuPy's <cupy/complex.cuh> so the reference kernels.cu
// compiles as plain C++ for the CPU (test infrastructure, oracle/ref_cpu).
#pragma once
#include <complex>
using std::complex;
using std::abs;
