// Shared device helpers for the RefSPI-MaxLP sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <atomic>

#include "rspi.h"

#define RSPI_FULL_MASK 0xffffffffu

// Launch-status check used by every C-ABI wrapper.
#define RSPI_RETURN_LAUNCH()                          \
    do {                                              \
        cudaError_t e_ = cudaGetLastError();          \
        return e_ == cudaSuccess ? RSPI_OK : RSPI_ERR_CUDA; \
    } while (0)

// First error wins; the caller reads the word after synchronising.
__device__ __forceinline__ void rspi_flag(int *err, int code) {
    if (err) atomicCAS(err, 0, code);
}

// IEEE double operations that the compiler may not contract into FMAs.  Used
// wherever an integer result (a pixel index, a floor or a rint) depends on
// the rounding of an expression, so it matches the FP64 restatement exactly.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }

// Row x and column y of pixel p = x * size + y (0 <= p < size^2, size <=
// 46340) without the integer division sequence: a float estimate of p / size
// (its error is far below one) and one exact correction step.
__device__ __forceinline__ void pixel_xy(int p, int size, float inv_size, int &x, int &y) {
    int q = (int)((float)p * inv_size);
    int r = p - q * size;
    if (r < 0) {
        --q;
        r += size;
    } else if (r >= size) {
        ++q;
        r -= size;
    }
    x = q;
    y = r;
}

// One rotated log-slice value (kernels.cu:19-41 with log_flag = 1, scale = 1):
// bilinear sample of the holographic slice w at R(angle)(p - cen) + cen, plus
// bg, then log; -1000 outside the detector or below 1e-20.  Shared by the
// slice kernel and the FP64 rescoring so both produce identical values.
__device__ __forceinline__ double rot_log_value(const double *__restrict__ w, int x, int y,
                                                int size, double ac, double as, double bg) {
    const int cen = size / 2;
    const double xc = (double)(x - cen), yc = (double)(y - cen);
    const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
    const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
    const double fxl = floor(tx), fyl = floor(ty);
    if (fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2) return -1000.;
    const int ix = (int)fxl, iy = (int)fyl;
    const double fx = tx - fxl, fy = ty - fyl;
    const double cx = 1. - fx, cy = 1. - fy;
    const double *r0 = w + (long long)ix * size + iy;
    const double *r1 = r0 + size;
    double v = xmul(xmul(r0[0], cx), cy);
    v = xadd(v, xmul(xmul(r1[0], fx), cy));
    v = xadd(v, xmul(xmul(r0[1], cx), fy));
    v = xadd(v, xmul(xmul(r1[1], fx), fy));
    v = xadd(v, bg);
    return v < 1.e-20 ? -1000. : log(v);
}

// Detector pixel of model pixel (tx, ty) for a frame with rotation (c, s):
// maxLP.py:250-252, x' = c qx + (-s) qy, y' = s qx + c qy, rint(x' size + size//2).
__device__ __forceinline__ void forward_pixel(int tx, int ty, double c, double s, int size,
                                              int &ox, int &oy) {
    const double ds = (double)size, c0 = (double)(size / 2);
    const double qx = ((double)tx - c0) / ds, qy = ((double)ty - c0) / ds;
    const double xr = xadd(xmul(c, qx), xmul(-s, qy));
    const double yr = xadd(xmul(s, qx), xmul(c, qy));
    ox = (int)rint(xadd(xmul(xr, ds), c0));
    oy = (int)rint(xadd(xmul(yr, ds), c0));
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(RSPI_FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ int warp_max_int(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(RSPI_FULL_MASK, v, o));
    return v;
}

// Argmax order of NumPy/CuPy: a NaN beats every number (the first NaN wins),
// otherwise the larger value wins and ties go to the smaller index.
__device__ __forceinline__ bool argmax_better(double a, int ia, double b, int ib) {
    bool na = isnan(a), nb = isnan(b);
    if (na || nb) {
        if (na && nb) return ia < ib;
        return na;
    }
    if (a != b) return a > b;
    return ia < ib;
}

// Block-wide sum of one double per thread; every thread gets the result.
// `scratch` holds >= 32 doubles.  Fixed reduction order (deterministic).
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double t = 0.;
    if (wid == 0) {
        t = lane < nw ? scratch[lane] : 0.;
        t = warp_sum(t);
        if (lane == 0) scratch[0] = t;
    }
    __syncthreads();
    t = scratch[0];
    __syncthreads();
    return t;
}

// Per-device host state: the library may drive several GPUs from one process,
// so every cached device property and kernel attribute is kept per device.
constexpr int RSPI_MAX_DEVICES = 64;

static inline int rspi_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

// SM count of the current device (cached per device).
static inline int rspi_sm_count() {
    static std::atomic<int> count[RSPI_MAX_DEVICES];
    const int dev = rspi_device();
    int c = (dev >= 0 && dev < RSPI_MAX_DEVICES) ? count[dev].load(std::memory_order_relaxed) : 0;
    if (c <= 0) {
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
        if (c <= 0) c = 148;
        if (dev >= 0 && dev < RSPI_MAX_DEVICES) count[dev].store(c, std::memory_order_relaxed);
    }
    return c;
}

// Dynamic shared-memory opt-in of one kernel, applied on each device the
// first time a launch there needs more than the default: one static
// RspiSmemOptIn per kernel instance.  Concurrent first calls on one device
// both apply the same attribute, which is harmless.  Returns false when the
// attribute cannot be set.
struct RspiSmemOptIn {
    std::atomic<size_t> done[RSPI_MAX_DEVICES];
};

static inline bool rspi_smem_optin(const void *kernel, size_t smem, RspiSmemOptIn &st) {
    const int dev = rspi_device();
    const bool cached = dev >= 0 && dev < RSPI_MAX_DEVICES;
    if (cached && st.done[dev].load(std::memory_order_acquire) >= smem) return true;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return false;
    if (cached) {
        size_t prev = st.done[dev].load(std::memory_order_relaxed);
        while (prev < smem &&
               !st.done[dev].compare_exchange_weak(prev, smem, std::memory_order_release))
            ;
    }
    return true;
}

static inline unsigned rspi_blocks(long long work, int threads, int cap_per_sm = 8) {
    long long b = (work + threads - 1) / threads;
    long long cap = (long long)rspi_sm_count() * cap_per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}
