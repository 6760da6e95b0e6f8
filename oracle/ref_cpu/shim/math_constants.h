// Host stand-in for CUDA's <math_constants.h>: only the constant kernels.cu uses.
#pragma once
#include <cmath>
#define CUDART_PI M_PI
