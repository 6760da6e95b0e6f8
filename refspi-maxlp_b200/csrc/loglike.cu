// Sparse-photon Poisson log-likelihood over frames x states (row a7).
//
// Replaces calc_prob_all (kernels.cu:116-137), which the reference launches
// once per (state, rotation) with one thread per frame walking its photon
// list.  Here one CTA owns a tile of T consecutive likelihood rows: it stages
// their rotated log-slices in shared memory (T * p_pad values), then every
// warp takes frames from a shared counter (frames pre-sorted by size, so the
// greedy order balances uneven photon counts) and walks the frame's packed
// entry rows.  In a row, lane b holds a photon whose sel index is b mod 32,
// so the warp's shared-memory gather hits 32 distinct banks.  Each lane
// accumulates count * L in FP64 for the T rows; a warp reduction finishes
// the frame and adds init[s0] * scale[d] (kernels.cu:126).
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;

template <typename TL, typename TO, int T>
__global__ void __launch_bounds__(1024)
k_loglike(const TL *__restrict__ lsl, long long p_pad, long long num_rot,
          const double *__restrict__ init, const double *__restrict__ scales,
          const unsigned int *__restrict__ entries, const long long *__restrict__ row_off,
          const int *__restrict__ frame_order, long long n_data, long long row_begin,
          long long row_end, TO *__restrict__ ll, long long ll_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TL *sl = reinterpret_cast<TL *>(smem_raw);
    __shared__ int next_frame;
    const int lane = threadIdx.x & 31;
    const long long n_rows = row_end - row_begin;
    const long long n_tiles = (n_rows + T - 1) / T;
    const int cmax = (int)p_pad - 1;  // entries never exceed it; the clamp keeps reads in bounds

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        // stage the tile's slices (16-byte vector copies; rows are contiguous)
        {
            const long long nvec = (long long)nt * p_pad * sizeof(TL) / 16;
            const int4 *src = reinterpret_cast<const int4 *>(lsl + (first - row_begin) * p_pad);
            int4 *dst = reinterpret_cast<int4 *>(sl);
            for (long long i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = src[i];
            const long long nzero = (long long)(T - nt) * p_pad * sizeof(TL) / 16;
            for (long long i = threadIdx.x; i < nzero; i += blockDim.x) dst[nvec + i] = int4{0, 0, 0, 0};
        }
        if (threadIdx.x == 0) next_frame = 0;
        __syncthreads();

        double ini[T];
#pragma unroll
        for (int t = 0; t < T; ++t) ini[t] = t < nt ? init[(first + t) / num_rot] : 0.;

        while (true) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&next_frame, 1);
            k = __shfl_sync(RSPI_FULL_MASK, k, 0);
            if (k >= n_data) break;
            const int d = frame_order ? frame_order[k] : k;
            const long long r0 = row_off[d], r1 = row_off[d + 1];
            double acc[T];
#pragma unroll
            for (int t = 0; t < T; ++t) acc[t] = 0.;
            const unsigned int *ep = entries + r0 * 32 + lane;
            long long r = r0;
            for (; r + 4 <= r1; r += 4, ep += 128) {
                unsigned e[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) e[u] = __ldg(ep + 32 * u);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int c = min((int)(e[u] >> 16), cmax);
                    const double cnt = (double)(e[u] & 0xffffu);
#pragma unroll
                    for (int t = 0; t < T; ++t) acc[t] = fma(cnt, (double)sl[t * p_pad + c], acc[t]);
                }
            }
            for (; r < r1; ++r, ep += 32) {
                const unsigned e = __ldg(ep);
                const int c = min((int)(e >> 16), cmax);
                const double cnt = (double)(e & 0xffffu);
#pragma unroll
                for (int t = 0; t < T; ++t) acc[t] = fma(cnt, (double)sl[t * p_pad + c], acc[t]);
            }
#pragma unroll
            for (int t = 0; t < T; ++t) acc[t] = warp_sum(acc[t]);
            if (lane < nt) {
                double v = 0.;
#pragma unroll
                for (int t = 0; t < T; ++t)
                    if (t == lane) v = ini[t] * scales[d] + acc[t];
                ll[(first + lane - row_begin) * ll_stride + d] = (TO)v;
            }
        }
        __syncthreads();
    }
}

template <typename TL, typename TO, int T>
int launch_t(const void *lsl, long long p_pad, long long num_rot, const double *init,
             const double *scales, const unsigned *entries, const long long *row_off,
             const int *frame_order, long long n_data, long long row_begin, long long row_end,
             void *ll, long long ll_stride, int warps, int n_ctas, cudaStream_t stream) {
    const size_t smem = (size_t)T * p_pad * sizeof(TL);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    auto kern = k_loglike<TL, TO, T>;
    static RspiSmemOptIn optin;   // once per device, so launches can be graph-captured
    if (!rspi_smem_optin((const void *)kern, smem, optin)) return RSPI_ERR_CUDA;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)((SMEM_LIMIT) / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    kern<<<n_ctas, warps * 32, smem, stream>>>(
        (const TL *)lsl, p_pad, num_rot, init, scales, entries, row_off, frame_order, n_data,
        row_begin, row_end, (TO *)ll, ll_stride);
    RSPI_RETURN_LAUNCH();
}

template <typename TL, typename TO>
int dispatch_t(int T, const void *lsl, long long p_pad, long long num_rot, const double *init,
               const double *scales, const unsigned *entries, const long long *row_off,
               const int *frame_order, long long n_data, long long row_begin, long long row_end,
               void *ll, long long ll_stride, int warps, int n_ctas, cudaStream_t stream) {
#define RSPI_LL_CASE(TT)                                                                     \
    case TT:                                                                                 \
        return launch_t<TL, TO, TT>(lsl, p_pad, num_rot, init, scales, entries, row_off,     \
                                    frame_order, n_data, row_begin, row_end, ll, ll_stride,  \
                                    warps, n_ctas, stream);
    switch (T) {
        RSPI_LL_CASE(1)
        RSPI_LL_CASE(2)
        RSPI_LL_CASE(3)
        RSPI_LL_CASE(4)
        RSPI_LL_CASE(6)
        RSPI_LL_CASE(8)
        default:
            return RSPI_ERR_ARG;
    }
#undef RSPI_LL_CASE
}

}  // namespace

extern "C" int rspi_loglike_max_tile(long long p_pad, int slice_dtype) {
    const long long bytes = p_pad * (slice_dtype == 1 ? 8 : 4);
    static const int tiles[] = {8, 6, 4, 3, 2, 1};
    for (int t : tiles)
        if (bytes * t <= SMEM_LIMIT - 1024) return t;
    return 0;
}

extern "C" int rspi_loglike(const void *lslices, int slice_dtype, long long p_pad,
                            long long num_rot, const double *init, const double *scales,
                            const unsigned int *entries, const long long *row_off,
                            const int *frame_order, long long n_data, long long row_begin,
                            long long row_end, void *ll, int out_dtype, long long ll_stride,
                            int states_per_tile, int warps_per_cta, int n_ctas,
                            cudaStream_t stream) {
    if (!lslices || !init || !scales || !entries || !row_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_pad <= 0 || p_pad % 32 || num_rot <= 0 || row_begin < 0 ||
        row_end < row_begin || ll_stride < n_data || warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0) return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    if (slice_dtype == 0 && out_dtype == 0)
        return dispatch_t<float, float>(states_per_tile, lslices, p_pad, num_rot, init, scales,
                                        entries, row_off, frame_order, n_data, row_begin,
                                        row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    if (slice_dtype == 0 && out_dtype == 1)
        return dispatch_t<float, double>(states_per_tile, lslices, p_pad, num_rot, init, scales,
                                         entries, row_off, frame_order, n_data, row_begin,
                                         row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    if (slice_dtype == 1 && out_dtype == 1)
        return dispatch_t<double, double>(states_per_tile, lslices, p_pad, num_rot, init, scales,
                                          entries, row_off, frame_order, n_data, row_begin,
                                          row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    if (slice_dtype == 1 && out_dtype == 0)
        return dispatch_t<double, float>(states_per_tile, lslices, p_pad, num_rot, init, scales,
                                         entries, row_off, frame_order, n_data, row_begin,
                                         row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    return RSPI_ERR_ARG;
}
