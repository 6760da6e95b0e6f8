// Screening likelihood, interleaved form (row a7, chosen form).
//
// The FP32 slices of a tile's T rows are staged in shared memory
// interleaved by pixel, sl[c*T + t], so one vector gather (8 bytes for T=2,
// 16 bytes for T=4) brings all T rows' values of a photon.  The photon
// entries are the 16-bit layout of rspi_ll16_entry_fill: lane b holds an
// index = b (mod 32); for the vector gathers a half (T=2) or a quarter (T=4)
// warp then touches distinct 8- or 16-byte banks, so the gathers stay
// conflict-free.  Indices are validated once on the host side of the
// pipeline (rspi_entries16_check), so the hot loop has no clamp.  Each warp
// streams a contiguous, word-balanced range of frames with a prefetch that
// crosses frame boundaries; loop indices are 32-bit.
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;
constexpr int PF = 8;

// Accumulators: T floats kept as float2 pairs so Blackwell's packed FP32x2
// add (FADD2) sums two rows per instruction.
template <int T>
struct Acc {
    static constexpr int NP = (T + 1) / 2;   // float2 pairs
    float2 p[NP];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < NP; ++i) p[i] = make_float2(0.f, 0.f);
    }
};

// One word's contribution (two photons, every row of the tile) and its add.
template <int T>
struct Contrib {
    float2 p[(T + 1) / 2];
};

template <int T>
__device__ __forceinline__ Contrib<T> gather_word(const unsigned char *sl, unsigned w);

template <>
__device__ __forceinline__ Contrib<1> gather_word<1>(const unsigned char *sl, unsigned w) {
    const float v0 = *reinterpret_cast<const float *>(sl + (w & 0xffffu) * 4u);
    const float v1 = *reinterpret_cast<const float *>(sl + (w >> 16) * 4u);
    Contrib<1> c;
    c.p[0] = make_float2(v0 + v1, 0.f);
    return c;
}
template <>
__device__ __forceinline__ Contrib<2> gather_word<2>(const unsigned char *sl, unsigned w) {
    const float2 v0 = *reinterpret_cast<const float2 *>(sl + (w & 0xffffu) * 8u);
    const float2 v1 = *reinterpret_cast<const float2 *>(sl + (w >> 16) * 8u);
    Contrib<2> c;
    c.p[0] = __fadd2_rn(v0, v1);
    return c;
}
template <>
__device__ __forceinline__ Contrib<4> gather_word<4>(const unsigned char *sl, unsigned w) {
    const float4 v0 = *reinterpret_cast<const float4 *>(sl + (w & 0xffffu) * 16u);
    const float4 v1 = *reinterpret_cast<const float4 *>(sl + (w >> 16) * 16u);
    Contrib<4> c;
    c.p[0] = __fadd2_rn(make_float2(v0.x, v0.y), make_float2(v1.x, v1.y));
    c.p[1] = __fadd2_rn(make_float2(v0.z, v0.w), make_float2(v1.z, v1.w));
    return c;
}

template <int T>
__device__ __forceinline__ void add_contrib(Acc<T> &a, const Contrib<T> &c) {
    if (T == 1) {
        a.p[0].x += c.p[0].x;
    } else {
#pragma unroll
        for (int i = 0; i < (T + 1) / 2; ++i) a.p[i] = __fadd2_rn(a.p[i], c.p[i]);
    }
}

template <int T>
__device__ __forceinline__ void add_word(Acc<T> &a, const unsigned char *sl, unsigned w);

template <>
__device__ __forceinline__ void add_word<1>(Acc<1> &a, const unsigned char *sl, unsigned w) {
    const float v0 = *reinterpret_cast<const float *>(sl + (w & 0xffffu) * 4u);
    const float v1 = *reinterpret_cast<const float *>(sl + (w >> 16) * 4u);
    a.p[0].x += v0 + v1;
}
template <>
__device__ __forceinline__ void add_word<2>(Acc<2> &a, const unsigned char *sl, unsigned w) {
    const float2 v0 = *reinterpret_cast<const float2 *>(sl + (w & 0xffffu) * 8u);
    const float2 v1 = *reinterpret_cast<const float2 *>(sl + (w >> 16) * 8u);
    a.p[0] = __fadd2_rn(a.p[0], __fadd2_rn(v0, v1));
}
template <>
__device__ __forceinline__ void add_word<4>(Acc<4> &a, const unsigned char *sl, unsigned w) {
    const float4 v0 = *reinterpret_cast<const float4 *>(sl + (w & 0xffffu) * 16u);
    const float4 v1 = *reinterpret_cast<const float4 *>(sl + (w >> 16) * 16u);
    a.p[0] = __fadd2_rn(a.p[0], __fadd2_rn(make_float2(v0.x, v0.y), make_float2(v1.x, v1.y)));
    a.p[1] = __fadd2_rn(a.p[1], __fadd2_rn(make_float2(v0.z, v0.w), make_float2(v1.z, v1.w)));
}

// Reduce-scatter over the warp: afterwards lane l holds the warp total of
// row (l mod T).  log2(T) exchange steps halve the values a lane carries,
// then 5 - log2(T) plain butterfly steps finish the sums.
template <int T>
__device__ __forceinline__ float reduce_scatter(Acc<T> &a, int lane);

template <>
__device__ __forceinline__ float reduce_scatter<1>(Acc<1> &a, int lane) {
    return warp_sum(a.p[0].x);
}
template <>
__device__ __forceinline__ float reduce_scatter<2>(Acc<2> &a, int lane) {
    const bool hi = lane & 1;
    float keep = hi ? a.p[0].y : a.p[0].x;
    const float send = hi ? a.p[0].x : a.p[0].y;
    keep += __shfl_xor_sync(RSPI_FULL_MASK, send, 1);
#pragma unroll
    for (int o = 2; o < 32; o <<= 1) keep += __shfl_xor_sync(RSPI_FULL_MASK, keep, o);
    return keep;
}
template <>
__device__ __forceinline__ float reduce_scatter<4>(Acc<4> &a, int lane) {
    // step 1 (xor 2): keep the pair of rows (lane >> 1) & 1
    const bool b1 = lane & 2;
    float2 keep = b1 ? a.p[1] : a.p[0];
    const float2 send = b1 ? a.p[0] : a.p[1];
    keep.x += __shfl_xor_sync(RSPI_FULL_MASK, send.x, 2);
    keep.y += __shfl_xor_sync(RSPI_FULL_MASK, send.y, 2);
    // step 2 (xor 1): keep row (lane & 1) of the pair
    const bool b0 = lane & 1;
    float k = b0 ? keep.y : keep.x;
    const float s = b0 ? keep.x : keep.y;
    k += __shfl_xor_sync(RSPI_FULL_MASK, s, 1);
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) k += __shfl_xor_sync(RSPI_FULL_MASK, k, o);
    return k;   // row (lane & 3)
}

template <int T>
__global__ void __launch_bounds__(T == 4 ? 512 : 1024)
k_screen_ll2(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const unsigned *__restrict__ words, const long long *__restrict__ row_off, int n_data,
             long long row_begin, long long row_end, float *__restrict__ ll, long long ll_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *slf = reinterpret_cast<float *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;

    // word-balanced frame range of this warp (word offsets = row offsets / 2)
    const int qtot = (int)(row_off[n_data] >> 1);
    auto lower = [&](int target) {
        int lo = 0, hi = n_data;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)(row_off[mid] >> 1) < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int fb = wid == 0 ? 0 : lower((int)((long long)qtot * wid / nw));
    const int fe = wid == nw - 1 ? n_data : lower((int)((long long)qtot * (wid + 1) / nw));

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        // stage and interleave: sl[c][t] = L[first + t][c]
        const float *src = lsl + (first - row_begin) * (long long)p_row;
        for (int i = threadIdx.x; i < T * p_row; i += blockDim.x) {
            const int t = i / p_row, c = i - t * p_row;
            slf[c * T + t] = t < nt ? __ldg(src + i) : 0.f;
        }
        __syncthreads();
        if (fb >= fe) continue;

        // this lane's row of the tile (stores go through lane < nt)
        const int my_t = lane & (T - 1);
        const double my_init = my_t < nt ? init[(first + my_t) / num_rot] : 0.;
        float *my_ll = ll + (first + my_t - row_begin) * ll_stride;
        Acc<T> acc;
        acc.zero();

        // frame offsets and scales of the next 32 frames, one per lane
        int base = fb;
        int my_end = fb + lane < n_data ? (int)(row_off[fb + lane + 1] >> 1) : 0x7fffffff;
        double my_scale = fb + lane < n_data ? scales[fb + lane] : 0.;
        int f = fb;
        int q = (int)(row_off[fb] >> 1);
        const int qend = (int)(row_off[fe] >> 1);
        int fend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
        auto finish = [&]() {
            const float tot = reduce_scatter<T>(acc, lane);
            const double sc = __shfl_sync(RSPI_FULL_MASK, my_scale, f - base);
            if (lane < nt) my_ll[f] = (float)(my_init * sc + (double)tot);
            acc.zero();
            ++f;
            if (f - base == 32) {
                base = f;
                my_end = f + lane < n_data ? (int)(row_off[f + lane + 1] >> 1) : 0x7fffffff;
                my_scale = f + lane < n_data ? scales[f + lane] : 0.;
            }
            fend = f < fe ? __shfl_sync(RSPI_FULL_MASK, my_end, f - base) : qend + 1;
        };
        while (f < fe && fend == q) finish();   // frames without photons

        const unsigned *wp = words + (long long)q * 32 + lane;
        unsigned cur[PF], nxt[PF];
#pragma unroll
        for (int k = 0; k < PF; ++k) cur[k] = q + k < qend ? __ldg(wp + 32 * k) : 0u;
        while (q < qend) {
            const int nb = min(PF, qend - q);
#pragma unroll
            for (int k = 0; k < PF; ++k) nxt[k] = q + PF + k < qend ? __ldg(wp + 32 * (PF + k)) : 0u;
            // gather phase without branches (slots past nb hold word 0: a
            // valid address whose contribution is never added)
            Contrib<T> cb[PF];
#pragma unroll
            for (int k = 0; k < PF; ++k) cb[k] = gather_word<T>(smem_raw, cur[k]);
#pragma unroll
            for (int k = 0; k < PF; ++k) {
                if (k < nb) {
                    add_contrib<T>(acc, cb[k]);
                    if (q + k + 1 == fend) {
                        finish();
                        while (f < fe && fend == q + k + 1) finish();
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PF; ++k) cur[k] = nxt[k];
            q += PF;
            wp += 32 * PF;
        }
    }
}

template <int T>
int launch2(const float *lsl, long long p_row, long long num_rot, const double *init,
            const double *scales, const unsigned *words, const long long *row_off,
            long long n_data, long long r0, long long r1, float *ll, long long stride, int warps,
            int n_ctas, cudaStream_t stream) {
    const size_t smem = (size_t)T * p_row * sizeof(float);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (r1 - r0 + T - 1) / T;
    if (T == 4) warps = min(warps, 16);   // register budget of the 4-row tile
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll2<T><<<n_ctas, warps * 32, smem, stream>>>(
        lsl, (int)p_row, (int)num_rot, init, scales, words, row_off, (int)n_data, r0, r1, ll,
        stride);
    RSPI_RETURN_LAUNCH();
}

// max entry index of a 16-bit entry array (validation before the clamp-free kernel)
__global__ void k_max_u16(const unsigned short *__restrict__ e, long long n,
                          unsigned *__restrict__ out) {
    unsigned m = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        m = max(m, (unsigned)e[i]);
    m = (unsigned)warp_max_int((int)m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace

extern "C" int rspi_entries16_check(const unsigned short *entries, long long n_entries,
                                    unsigned *max_index, cudaStream_t stream) {
    if (!entries || !max_index || n_entries < 0) return RSPI_ERR_ARG;
    cudaMemsetAsync(max_index, 0, sizeof(unsigned), stream);
    if (n_entries > 0)
        k_max_u16<<<rspi_blocks(n_entries, 256), 256, 0, stream>>>(entries, n_entries, max_index);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_screen_loglike2(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned short *entries, const long long *row_off,
                                    long long n_data, long long row_begin, long long row_end,
                                    float *ll, long long ll_stride, int states_per_tile,
                                    int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !entries || !row_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin || ll_stride < n_data ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(entries) & 3) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const unsigned *w = reinterpret_cast<const unsigned *>(entries);
    switch (states_per_tile) {
        case 1:
            return launch2<1>(lslices, p_row, num_rot, init, scales, w, row_off, n_data,
                              row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
        case 2:
            return launch2<2>(lslices, p_row, num_rot, init, scales, w, row_off, n_data,
                              row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
        case 4:
            return launch2<4>(lslices, p_row, num_rot, init, scales, w, row_off, n_data,
                              row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
        default:
            return RSPI_ERR_ARG;
    }
}
