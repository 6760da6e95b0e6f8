// Streaming likelihood kernel (row a7), both forms.
//
// Same work as k_loglike / k_screen_ll (one CTA per tile of T likelihood
// rows, slices staged in shared memory, bank-conflict-free packed entries)
// with a different frame schedule: the packed entry words of all frames are
// one contiguous stream, and each warp owns a contiguous range of frames
// holding ~1/W of the words (split once per CTA by binary search on the
// word offsets).  A warp streams its range in batches of PF words, loading
// the next batch while it processes the current one, across frame
// boundaries, so there is no per-frame load bubble and no shared counter.
// Per lane the words of a frame are consumed in order and the warp
// reduction is the same as in k_loglike, so the FP64 form's values are
// bit-identical to it (and to the FP64 rescoring in screen.cu).
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;
constexpr int PF = 8;   // words per prefetch batch

// 32-bit (sel << 16 | count) entries, FP64 slices, FP64 sums: one row per word
struct FormF64 {
    using TL = double;
    using Acc = double;
    using TO = double;
    static constexpr int WORD_SHIFT = 0;  // words = rows
    template <int T>
    __device__ __forceinline__ static void add(Acc (&acc)[T], const TL *sl, long long p_row,
                                               unsigned w, unsigned cmax) {
        const unsigned c = min(w >> 16, cmax);
        const double cnt = (double)(w & 0xffffu);
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = fma(cnt, sl[t * p_row + c], acc[t]);
    }
};

// 16-bit sel indices, counts expanded, two rows per word; FP32 slices and sums
struct FormScreen {
    using TL = float;
    using Acc = float;
    using TO = float;
    static constexpr int WORD_SHIFT = 1;  // words = rows / 2
    template <int T>
    __device__ __forceinline__ static void add(Acc (&acc)[T], const TL *sl, long long p_row,
                                               unsigned w, unsigned cmax) {
        const unsigned c0 = min(w & 0xffffu, cmax), c1 = min(w >> 16, cmax);
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] += sl[t * p_row + c0] + sl[t * p_row + c1];
    }
};

template <class F, int T>
__device__ __forceinline__ void finish_frame(typename F::Acc (&acc)[T], long long d, int lane,
                                             int nt, const double (&ini)[T],
                                             const double *__restrict__ scales,
                                             typename F::TO *__restrict__ ll, long long first,
                                             long long row_begin, long long ll_stride) {
#pragma unroll
    for (int t = 0; t < T; ++t) acc[t] = warp_sum(acc[t]);
    if (lane < nt) {
        double v = 0.;
#pragma unroll
        for (int t = 0; t < T; ++t)
            if (t == lane) v = ini[t] * scales[d] + (double)acc[t];
        ll[(first + lane - row_begin) * ll_stride + d] = (typename F::TO)v;
    }
#pragma unroll
    for (int t = 0; t < T; ++t) acc[t] = 0;
}

// larger tiles need more registers per thread: cap the CTA at 512 threads
template <int T>
constexpr int max_threads() { return T > 2 ? 512 : 1024; }

template <class F, int T>
__global__ void __launch_bounds__(max_threads<T>())
k_ll_stream(const typename F::TL *__restrict__ lsl, long long p_row, long long num_rot,
            const double *__restrict__ init, const double *__restrict__ scales,
            const unsigned *__restrict__ words, const long long *__restrict__ row_off,
            long long n_data, long long row_begin, long long row_end,
            typename F::TO *__restrict__ ll, long long ll_stride) {
    using TL = typename F::TL;
    using Acc = typename F::Acc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TL *sl = reinterpret_cast<TL *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned cmax = (unsigned)p_row - 1;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;

    // this warp's frames [fb, fe): balanced by words, fixed for every tile
    const long long qtot = row_off[n_data] >> F::WORD_SHIFT;
    auto lower = [&](long long target) {
        long long lo = 0, hi = n_data;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if ((row_off[mid] >> F::WORD_SHIFT) < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const long long fb = wid == 0 ? 0 : lower(qtot * wid / nw);
    const long long fe = wid == nw - 1 ? n_data : lower(qtot * (wid + 1) / nw);

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();  // previous tile's readers are done
        {
            const long long nvec = (long long)nt * p_row * sizeof(TL) / 16;
            const int4 *src = reinterpret_cast<const int4 *>(lsl + (first - row_begin) * p_row);
            int4 *dst = reinterpret_cast<int4 *>(sl);
            for (long long i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = src[i];
            const long long nzero = (long long)(T - nt) * p_row * sizeof(TL) / 16;
            for (long long i = threadIdx.x; i < nzero; i += blockDim.x) dst[nvec + i] = int4{0, 0, 0, 0};
        }
        __syncthreads();
        if (fb >= fe) continue;

        double ini[T];
#pragma unroll
        for (int t = 0; t < T; ++t) ini[t] = t < nt ? init[(first + t) / num_rot] : 0.;
        Acc acc[T];
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0;

        long long f = fb;
        long long fend = row_off[f + 1] >> F::WORD_SHIFT;   // first word after frame f
        long long q = row_off[fb] >> F::WORD_SHIFT;
        const long long qend = row_off[fe] >> F::WORD_SHIFT;
        // frames with no words before the first word
        while (f < fe && fend == q) {
            finish_frame<F, T>(acc, f, lane, nt, ini, scales, ll, first, row_begin, ll_stride);
            ++f;
            if (f < fe) fend = row_off[f + 1] >> F::WORD_SHIFT;
        }
        unsigned cur[PF], nxt[PF];
#pragma unroll
        for (int k = 0; k < PF; ++k)
            cur[k] = q + k < qend ? __ldg(words + (q + k) * 32 + lane) : 0u;
        while (q < qend) {
#pragma unroll
            for (int k = 0; k < PF; ++k)
                nxt[k] = q + PF + k < qend ? __ldg(words + (q + PF + k) * 32 + lane) : 0u;
#pragma unroll
            for (int k = 0; k < PF; ++k) {
                if (q + k < qend) {
                    F::template add<T>(acc, sl, p_row, cur[k], cmax);
                    // close every frame that ends here (and empty ones after it)
                    while (f < fe && fend == q + k + 1) {
                        finish_frame<F, T>(acc, f, lane, nt, ini, scales, ll, first, row_begin,
                                           ll_stride);
                        ++f;
                        if (f < fe) fend = row_off[f + 1] >> F::WORD_SHIFT;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PF; ++k) cur[k] = nxt[k];
            q += PF;
        }
    }
}

template <class F, int T>
int launch(const void *lsl, long long p_row, long long num_rot, const double *init,
           const double *scales, const unsigned *words, const long long *row_off,
           long long n_data, long long r0, long long r1, void *ll, long long stride, int warps,
           int n_ctas, cudaStream_t stream) {
    const size_t smem = (size_t)T * p_row * sizeof(typename F::TL);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static RspiSmemOptIn optin;
    if (!rspi_smem_optin((const void *)k_ll_stream<F, T>, smem, optin)) return RSPI_ERR_CUDA;
    const long long n_tiles = (r1 - r0 + T - 1) / T;
    warps = min(warps, max_threads<T>() / 32);
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_ll_stream<F, T><<<n_ctas, warps * 32, smem, stream>>>(
        (const typename F::TL *)lsl, p_row, num_rot, init, scales, words, row_off, n_data, r0,
        r1, (typename F::TO *)ll, stride);
    RSPI_RETURN_LAUNCH();
}

template <class F>
int dispatch(int T, const void *lsl, long long p_row, long long num_rot, const double *init,
             const double *scales, const unsigned *words, const long long *row_off,
             long long n_data, long long r0, long long r1, void *ll, long long stride, int warps,
             int n_ctas, cudaStream_t stream) {
#define RSPI_ST(TT)                                                                            \
    case TT:                                                                                   \
        return launch<F, TT>(lsl, p_row, num_rot, init, scales, words, row_off, n_data, r0,    \
                             r1, ll, stride, warps, n_ctas, stream);
    switch (T) {
        RSPI_ST(1)
        RSPI_ST(2)
        RSPI_ST(3)
        RSPI_ST(4)
        RSPI_ST(6)
        RSPI_ST(8)
        default:
            return RSPI_ERR_ARG;
    }
#undef RSPI_ST
}

}  // namespace

extern "C" int rspi_loglike_stream(int form, const void *lslices, long long p_row,
                                   long long num_rot, const double *init, const double *scales,
                                   const void *entries, const long long *row_off,
                                   long long n_data, long long row_begin, long long row_end,
                                   void *ll, long long ll_stride, int states_per_tile,
                                   int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !entries || !row_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_row <= 0 || p_row % 32 || p_row > 65536 || num_rot <= 0 ||
        row_begin < 0 || row_end < row_begin || ll_stride < n_data || warps_per_cta < 1 ||
        warps_per_cta > 32 || (form != 0 && form != 1))
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(entries) & 3) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const unsigned *w = reinterpret_cast<const unsigned *>(entries);
    if (form == 1)
        return dispatch<FormF64>(states_per_tile, lslices, p_row, num_rot, init, scales, w,
                                 row_off, n_data, row_begin, row_end, ll, ll_stride,
                                 warps_per_cta, n_ctas, stream);
    return dispatch<FormScreen>(states_per_tile, lslices, p_row, num_rot, init, scales, w,
                                row_off, n_data, row_begin, row_end, ll, ll_stride,
                                warps_per_cta, n_ctas, stream);
}
