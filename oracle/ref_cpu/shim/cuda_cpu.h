// Force-included before the reference kernels.cu when it is compiled for the
// CPU: CUDA built-ins become host equivalents, and a kernel becomes a plain
// function that the launchers in launch.cpp call once per (block, thread).
// Test infrastructure only.
#pragma once
#include <cmath>
#include <algorithm>
struct rspi_cpu_dim3 { unsigned int x, y, z; };
extern thread_local rspi_cpu_dim3 threadIdx, blockIdx, blockDim, gridDim;
#define __global__
#define __device__
static inline int __double2int_rd(double x) { return (int)std::floor(x); }
static inline int __double2int_rn(double x) { return (int)std::nearbyint(x); }
static inline double atomicAdd(double *a, double v) { double o = *a; *a = o + v; return o; }
using std::min;
using std::max;
