// Per-frame reduction over states (rows a8, a9): first-index max/argmax
// (emc.py:207-209, prob.max(0) / prob.argmax(0)) and the FP64 log-sum-exp
// that normalises the posterior.  A CTA covers 32 frames (threadIdx.x) and
// splits the state axis over its warps (threadIdx.y); reads of LL[r][d0..d0+31]
// are coalesced.  Each thread keeps an online (max, argmax, sum exp(x-max));
// partial triples merge in a fixed order.
#include "rspi_common.cuh"

namespace {

constexpr int RY = 32;

struct Acc {
    double m;
    double s;
    int i;
};

template <bool LSE>
__device__ __forceinline__ void acc_push(Acc &a, double v, int r) {
    if (a.i < 0) {
        a = Acc{v, 1., r};
        return;
    }
    if (argmax_better(v, r, a.m, a.i)) {
        if (LSE) a.s = isnan(v) || isnan(a.m) ? a.s + 1. : a.s * exp(a.m - v) + 1.;
        a.m = v;
        a.i = r;
    } else if (LSE) {
        a.s += isnan(a.m) ? 1. : exp(v - a.m);
    }
}

__device__ __forceinline__ Acc acc_merge(Acc a, Acc b) {
    if (a.i < 0) return b;
    if (b.i < 0) return a;
    if (argmax_better(b.m, b.i, a.m, a.i)) {
        Acc t = a;
        a = b;
        b = t;
    }
    a.s = a.s + b.s * exp(b.m - a.m);
    return a;
}

template <typename TL, bool LSE>
__global__ void __launch_bounds__(32 * RY)
k_frame_reduce(const TL *__restrict__ ll, long long n_rows, long long n_data,
               double *__restrict__ maxll, int *__restrict__ rmax, double *__restrict__ logz) {
    __shared__ double sm[RY][33];
    __shared__ double ss[RY][33];
    __shared__ int si[RY][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long d = (long long)blockIdx.x * 32 + tx;
    Acc a{0., 0., -1};
    if (d < n_data) {
        // eight rows' loads in flight per thread, pushed in row order
        long long r = ty;
        for (; r + 7 * RY < n_rows; r += 8 * RY) {
            TL v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = __ldg(&ll[(r + u * RY) * n_data + d]);
#pragma unroll
            for (int u = 0; u < 8; ++u) acc_push<LSE>(a, (double)v[u], (int)(r + u * RY));
        }
        for (; r < n_rows; r += RY) acc_push<LSE>(a, (double)ll[r * n_data + d], (int)r);
    }
    sm[ty][tx] = a.m;
    ss[ty][tx] = a.s;
    si[ty][tx] = a.i;
    __syncthreads();
    if (ty == 0 && d < n_data) {
        Acc b{sm[0][tx], ss[0][tx], si[0][tx]};
        for (int k = 1; k < RY; ++k) b = acc_merge(b, Acc{sm[k][tx], ss[k][tx], si[k][tx]});
        if (maxll) maxll[d] = b.m;
        if (rmax) rmax[d] = b.i;
        if (logz) logz[d] = b.m + log(b.s);
    }
}

}  // namespace

extern "C" int rspi_frame_reduce(const void *ll, int ll_dtype, long long n_rows,
                                 long long n_data, double *maxll, int *rmax, double *logz,
                                 cudaStream_t stream) {
    if (!ll || n_rows <= 0 || n_data <= 0 || n_rows > 0x7fffffffLL) return RSPI_ERR_ARG;
    const dim3 block(32, RY);
    const unsigned grid = (unsigned)((n_data + 31) / 32);
    if (ll_dtype == 1 && logz)
        k_frame_reduce<double, true><<<grid, block, 0, stream>>>((const double *)ll, n_rows,
                                                                 n_data, maxll, rmax, logz);
    else if (ll_dtype == 1)
        k_frame_reduce<double, false><<<grid, block, 0, stream>>>((const double *)ll, n_rows,
                                                                  n_data, maxll, rmax, logz);
    else if (ll_dtype == 0 && logz)
        k_frame_reduce<float, true><<<grid, block, 0, stream>>>((const float *)ll, n_rows, n_data,
                                                                maxll, rmax, logz);
    else if (ll_dtype == 0)
        k_frame_reduce<float, false><<<grid, block, 0, stream>>>((const float *)ll, n_rows,
                                                                 n_data, maxll, rmax, logz);
    else
        return RSPI_ERR_ARG;
    RSPI_RETURN_LAUNCH();
}
