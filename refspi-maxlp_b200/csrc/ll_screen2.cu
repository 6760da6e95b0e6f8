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
#include <cuda_fp16.h>

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

// Reduce-scatter over the warp: afterwards lane l holds the warp total of
// row (l mod T).  log2(T) exchange steps halve the values a lane carries,
// then 5 - log2(T) plain butterfly steps finish the sums.
// Stage T consecutive slice rows into the interleaved tile sl[c][t]
// (column c of row t at c * T + t, zeros for rows past nt): each thread takes
// whole columns, T coalesced loads each, four columns' loads in flight.
template <int T>
__device__ __forceinline__ void stage_tile(float *sl, const float *__restrict__ src, int p_row,
                                           int nt) {
#pragma unroll 4
    for (int c = threadIdx.x; c < p_row; c += blockDim.x) {
        float v[T];
#pragma unroll
        for (int t = 0; t < T; ++t) v[t] = t < nt ? __ldg(src + (long long)t * p_row + c) : 0.f;
        if constexpr (T == 1) {
            sl[c] = v[0];
        } else if constexpr (T == 2) {
            reinterpret_cast<float2 *>(sl)[c] = make_float2(v[0], v[1]);
        } else {
#pragma unroll
            for (int t = 0; t < T; ++t) sl[c * T + t] = v[t];
        }
    }
}

template <int T>
__device__ __forceinline__ void stage_tile_h(__half *sl, const __half *__restrict__ src, int p_row,
                                             int nt) {
    const __half hz = __float2half(0.f);
#pragma unroll 4
    for (int c = threadIdx.x; c < p_row; c += blockDim.x) {
#pragma unroll
        for (int t = 0; t < T; ++t) sl[c * T + t] = t < nt ? src[(long long)t * p_row + c] : hz;
    }
}

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
        stage_tile<T>(slf, src, p_row, nt);
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

// Frame-at-a-time form of the same sums (the default for T = 1, 2): the
// warp walks its frames one by one; the first PFW words of each frame were
// loaded while the previous frame was summed, and a frame's sum runs without
// any per-word frame-boundary test.  Words past the frame's end are replaced
// by the lane's zero-column pair, which adds exactly 0.  Two accumulators
// per lane alternate between words.  Each value passes through at most
// (words + 8) FP32 roundings, within the screening bound.
template <int T, int PFW>
__global__ void __launch_bounds__(1024)
k_screen_ll3(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const unsigned *__restrict__ words, const long long *__restrict__ row_off, int n_data,
             long long row_begin, long long row_end, float *__restrict__ ll, long long ll_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *slf = reinterpret_cast<float *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
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
    const unsigned zc = (unsigned)(p_row - 32 + lane);
    const unsigned zpair = zc | (zc << 16);
    const int last = qtot - 1;   // last word index (-1: no words at all)
    auto word_at = [&](int q) -> unsigned {
        return last >= 0 ? __ldg(words + (long long)min(q, last) * 32 + lane) : zpair;
    };

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        const float *src = lsl + (first - row_begin) * (long long)p_row;
        stage_tile<T>(slf, src, p_row, nt);
        __syncthreads();
        if (fb >= fe) continue;

        const int my_t = lane & (T - 1);
        const double my_init = my_t < nt ? init[(first + my_t) / num_rot] : 0.;
        float *my_ll = ll + (first + my_t - row_begin) * ll_stride;
        int base = fb;
        int my_end = fb + lane < n_data ? (int)(row_off[fb + lane + 1] >> 1) : 0x7fffffff;
        double my_scale = fb + lane < n_data ? scales[fb + lane] : 0.;
        int q = (int)(row_off[fb] >> 1);
        unsigned pre[PFW];
#pragma unroll
        for (int k = 0; k < PFW; ++k) pre[k] = word_at(q + k);
        for (int f = fb; f < fe; ++f) {
            const int qe = __shfl_sync(RSPI_FULL_MASK, my_end, f - base);
            const int n = qe - q;
            unsigned cur[PFW];
#pragma unroll
            for (int k = 0; k < PFW; ++k) {
                cur[k] = k < n ? pre[k] : zpair;
                pre[k] = word_at(qe + k);          // the next frame's first words
            }
            Acc<T> a0, a1;
            a0.zero();
            a1.zero();
#pragma unroll
            for (int k = 0; k < PFW; k += 2) {
                add_contrib<T>(a0, gather_word<T>(smem_raw, cur[k]));
                add_contrib<T>(a1, gather_word<T>(smem_raw, cur[k + 1]));
            }
            for (int q2 = q + PFW; q2 < qe; q2 += 4) {   // frames longer than PFW words
                unsigned w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = q2 + k < qe ? word_at(q2 + k) : zpair;
                add_contrib<T>(a0, gather_word<T>(smem_raw, w[0]));
                add_contrib<T>(a1, gather_word<T>(smem_raw, w[1]));
                add_contrib<T>(a0, gather_word<T>(smem_raw, w[2]));
                add_contrib<T>(a1, gather_word<T>(smem_raw, w[3]));
            }
            Contrib<T> c1;
#pragma unroll
            for (int i = 0; i < (T + 1) / 2; ++i) c1.p[i] = a1.p[i];
            add_contrib<T>(a0, c1);
            const float tot = reduce_scatter<T>(a0, lane);
            const double sc = __shfl_sync(RSPI_FULL_MASK, my_scale, f - base);
            if (lane < nt) my_ll[f] = (float)(my_init * sc + (double)tot);
            q = qe;
            if (f + 1 - base == 32) {
                base = f + 1;
                my_end = base + lane < n_data ? (int)(row_off[base + lane + 1] >> 1) : 0x7fffffff;
                my_scale = base + lane < n_data ? scales[base + lane] : 0.;
            }
        }
    }
}

template <int T, int PFW>
int launch3(const float *lsl, long long p_row, long long num_rot, const double *init,
            const double *scales, const unsigned *words, const long long *row_off,
            long long n_data, long long r0, long long r1, float *ll, long long stride, int warps,
            int n_ctas, cudaStream_t stream) {
    const size_t smem = (size_t)T * p_row * sizeof(float);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll3<T, PFW>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (r1 - r0 + T - 1) / T;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll3<T, PFW><<<n_ctas, warps * 32, smem, stream>>>(
        lsl, (int)p_row, (int)num_rot, init, scales, words, row_off, (int)n_data, r0, r1, ll,
        stride);
    RSPI_RETURN_LAUNCH();
}

// ---------------------------------------------------------------------------
// Wide-entry form: 32-bit entries that already hold the byte offset of the
// photon's value in the interleaved tile (sel * 4T), four rows of a lane in
// one 16-byte group, so a lane issues one LDG.128 per four photons and each
// photon costs one shared gather and half a packed add.  Rows of a frame are
// padded to a multiple of four with the lane's zero column.
// ---------------------------------------------------------------------------
__global__ void k_wide_groups(const long long *__restrict__ row_off16, long long n,
                              int *__restrict__ groups) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride)
        groups[d] = (int)((row_off16[d + 1] - row_off16[d] + 3) >> 2);
}

__global__ void k_wide_fill(const unsigned short *__restrict__ ent16,
                            const long long *__restrict__ row_off16, long long n, int p_zero,
                            int tile, const long long *__restrict__ goff,
                            unsigned *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned scale = 4u * (unsigned)tile;
    for (long long d = warp; d < n; d += nwarp) {
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        const long long g0 = goff[d], ng = goff[d + 1] - g0;
        for (long long r = 0; r < 4 * ng; ++r) {
            unsigned v = (unsigned)(p_zero + lane);
            if (r < nr) {
                const long long rr = r0 + r;
                v = ent16[(rr >> 1) * 64 + lane * 2 + (rr & 1)];
            }
            out[((g0 + (r >> 2)) * 32 + lane) * 4 + (r & 3)] = v * scale;
        }
    }
}

// Bank-class layout of the wide entries.  A lane's shared gather at byte
// offset sel * B (B = 4, 8 bytes per pixel) falls in bank class sel mod C,
// C = 128 / B (the 32 four-byte banks taken B/4 at a time).  Here lane l only
// ever holds photons of class l mod C (and its zero column p_zero + l, of the
// same class since p_zero % 32 == 0), so the 32 addresses of every gather
// instruction fall in distinct bank classes, two lanes per class when C = 16,
// and the gather needs the minimum number of shared-memory wavefronts.  The
// k-th photon of class c goes to lane c + C (k mod 32/C), slot k / (32/C);
// a frame takes ceil(max_c n_c / (4 * 32/C)) groups.
constexpr int BANK_WARPS = 8;

__device__ __forceinline__ unsigned entry16_at(const unsigned short *__restrict__ ent16,
                                               long long rr, int lane) {
    return ent16[(rr >> 1) * 64 + lane * 2 + (rr & 1)];
}

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_wide_groups_banked(const unsigned short *__restrict__ ent16,
                     const long long *__restrict__ row_off16, long long n, int p_zero,
                     int classes, int slots, int *__restrict__ groups) {
    __shared__ int cnt[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n; d += nwarp) {
        cnt[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e % (unsigned)classes) : classes;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < classes && lane == __ffs(m) - 1) cnt[w][key] += __popc(m);
            __syncwarp();
        }
        int mx = lane < classes ? cnt[w][lane] : 0;
        mx = warp_max_int(mx);
        if (lane == 0) groups[d] = (mx + slots - 1) / slots;
        __syncwarp();
    }
}

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_wide_fill_banked(const unsigned short *__restrict__ ent16,
                   const long long *__restrict__ row_off16, long long n, int p_zero, int classes,
                   unsigned scale, const long long *__restrict__ goff,
                   unsigned *__restrict__ out) {
    __shared__ int base[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const int per = 32 / classes;
    const unsigned lt = (1u << lane) - 1u;
    for (long long d = warp; d < n; d += nwarp) {
        const long long g0 = goff[d], ng = goff[d + 1] - g0;
        // every slot of the frame starts as the lane's zero column
        const unsigned pad = (unsigned)(p_zero + lane) * scale;
        for (long long g = 0; g < ng; ++g)
            reinterpret_cast<uint4 *>(out)[(g0 + g) * 32 + lane] = make_uint4(pad, pad, pad, pad);
        base[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e % (unsigned)classes) : classes;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < classes) {
                const int k = base[w][key] + __popc(m & lt);
                const int slot_lane = key + classes * (k % per);
                const long long slot = k / per;
                if ((slot >> 2) < ng)
                    out[((g0 + (slot >> 2)) * 32 + slot_lane) * 4 + (slot & 3)] = e * scale;
            }
            __syncwarp();
            if (key < classes && lane == __ffs(m) - 1) base[w][key] += __popc(m);
            __syncwarp();
        }
    }
}

// Frame pairs: the two half-warps take the two frames of a pair, so one
// pass of the per-frame reduction and store serves two frames.  Two rows per
// tile (C = 16 bank classes); lane 16 h + c of a pair group holds frame h's
// photons of class c, four 16-bit q per group (column 16 q + c), the k-th
// photon of class c in slot k of that lane; a pair takes the larger of its
// frames' group counts ceil(max_c n_c / 4); every other slot holds the lane's
// zero column (q = (p_zero + lane) / 16, of class lane mod 16).
__global__ void k_pair_pad(long long n_slots, int p_zero, uint2 *__restrict__ out) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_slots;
         i += stride) {
        const unsigned pad = (unsigned)(p_zero + (int)(i & 31)) / 16u;
        const unsigned pad2 = pad | (pad << 16);
        out[i] = make_uint2(pad2, pad2);
    }
}

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_pair_fill(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
            long long n, int p_zero, const int *__restrict__ pair_slot,
            const long long *__restrict__ pgoff, unsigned short *__restrict__ out) {
    __shared__ int base[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (long long d = warp; d < n; d += nwarp) {
        const int ps = pair_slot[d];
        const long long p = ps >> 1;
        const int h = ps & 1;
        const long long g0 = pgoff[p], ng = pgoff[p + 1] - g0;
        base[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e % 16u) : 16;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < 16) {
                const int k = base[w][key] + __popc(m & lt);
                if ((k >> 2) < ng)
                    out[((g0 + (k >> 2)) * 32 + 16 * h + key) * 4 + (k & 3)] =
                        (unsigned short)(e / 16u);
            }
            __syncwarp();
            if (key < 16 && lane == __ffs(m) - 1) base[w][key] += __popc(m);
            __syncwarp();
        }
    }
}

// Frame quads: eight lanes per frame, four frames per warp.  Sub-frame u of
// a quad takes lanes 8 u + j (j < 8); lane j holds the frame's photons of
// bank classes j and j + 8, the one in slots 0 and 2 of a group (phase 0)
// and the other in slots 1 and 3 (phase 1), with the phases swapped on odd
// u: every shared gather of a half-warp then touches 16 distinct bank
// classes.  The k-th photon of class c goes to group k / 2, slot
// 2 (k mod 2) + phase; a quad takes the largest of its frames' group counts
// ceil(max_c n_c / 2); every other slot holds column p_zero + class (q =
// p_zero / 16), a zero column of the slot's class.
__global__ void k_quad_pad(long long n_slots, int p_zero, uint2 *__restrict__ out) {
    const unsigned pad = (unsigned)p_zero / 16u;
    const unsigned pad2 = pad | (pad << 16);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_slots;
         i += stride)
        out[i] = make_uint2(pad2, pad2);
}

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_quad_fill(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
            long long n, int p_zero, const int *__restrict__ quad_slot,
            const long long *__restrict__ qgoff, unsigned short *__restrict__ out) {
    __shared__ int base[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (long long d = warp; d < n; d += nwarp) {
        const int qs = quad_slot[d];
        const long long qd = qs >> 2;
        const int u = qs & 3;
        const long long g0 = qgoff[qd], ng = qgoff[qd + 1] - g0;
        base[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e % 16u) : 16;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < 16) {
                const int k = base[w][key] + __popc(m & lt);
                const int phase = (key >> 3) ^ (u & 1);
                if ((k >> 1) < ng)
                    out[((g0 + (k >> 1)) * 32 + 8 * u + (key & 7)) * 4 + 2 * (k & 1) + phase] =
                        (unsigned short)(e / 16u);
            }
            __syncwarp();
            if (key < 16 && lane == __ffs(m) - 1) base[w][key] += __popc(m);
            __syncwarp();
        }
    }
}

// The bank-class layout with 16-bit entries: lane l's photons all have
// class c = l mod C, so the tile column is sel = C q + c and the entry
// stores q (< 4096); the gather's byte offset is q * 128 + 4T (l mod C).
// Same slots and groups as k_wide_fill_banked, half the bytes.
__global__ void __launch_bounds__(BANK_WARPS * 32)
k_narrow_fill_banked(const unsigned short *__restrict__ ent16,
                     const long long *__restrict__ row_off16, long long n, int p_zero,
                     int classes, const long long *__restrict__ goff,
                     unsigned short *__restrict__ out) {
    __shared__ int base[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const int per = 32 / classes;
    const unsigned lt = (1u << lane) - 1u;
    for (long long d = warp; d < n; d += nwarp) {
        const long long g0 = goff[d], ng = goff[d + 1] - g0;
        const unsigned short pad = (unsigned short)((unsigned)(p_zero + lane) / (unsigned)classes);
        const unsigned pad2 = (unsigned)pad | ((unsigned)pad << 16);
        for (long long g = 0; g < ng; ++g)
            reinterpret_cast<uint2 *>(out)[(g0 + g) * 32 + lane] = make_uint2(pad2, pad2);
        base[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e % (unsigned)classes) : classes;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < classes) {
                const int k = base[w][key] + __popc(m & lt);
                const int slot_lane = key + classes * (k % per);
                const long long slot = k / per;
                if ((slot >> 2) < ng)
                    out[((g0 + (slot >> 2)) * 32 + slot_lane) * 4 + (slot & 3)] =
                        (unsigned short)(e / (unsigned)classes);
            }
            __syncwarp();
            if (key < classes && lane == __ffs(m) - 1) base[w][key] += __popc(m);
            __syncwarp();
        }
    }
}

template <int T>
__device__ __forceinline__ Contrib<T> gather_pair(const unsigned char *sl, unsigned a,
                                                  unsigned b) {
    Contrib<T> c;
    if (T == 1) {
        c.p[0] = make_float2(*reinterpret_cast<const float *>(sl + a) +
                                 *reinterpret_cast<const float *>(sl + b),
                             0.f);
    } else {
        const float2 v0 = *reinterpret_cast<const float2 *>(sl + a);
        const float2 v1 = *reinterpret_cast<const float2 *>(sl + b);
        c.p[0] = __fadd2_rn(v0, v1);
    }
    return c;
}

// One group of four photons of a lane: 32-bit entries hold the byte
// offsets; 16-bit entries hold q with offset q * 128 + lane_off.
template <int T>
__device__ __forceinline__ void gather_group(const unsigned char *sl, const uint4 &g, unsigned,
                                             Contrib<T> &c0, Contrib<T> &c1) {
    c0 = gather_pair<T>(sl, g.x, g.y);
    c1 = gather_pair<T>(sl, g.z, g.w);
}

template <int T>
__device__ __forceinline__ void gather_group(const unsigned char *sl, const uint2 &g,
                                             unsigned lane_off, Contrib<T> &c0, Contrib<T> &c1) {
    c0 = gather_pair<T>(sl, (g.x & 0xffffu) * 128u + lane_off, (g.x >> 16) * 128u + lane_off);
    c1 = gather_pair<T>(sl, (g.y & 0xffffu) * 128u + lane_off, (g.y >> 16) * 128u + lane_off);
}

template <bool NARROW> struct GroupOf { using type = uint4; };
template <> struct GroupOf<true> { using type = uint2; };

template <int T, bool NARROW>
__global__ void __launch_bounds__(1024)
k_screen_ll4(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const typename GroupOf<NARROW>::type *__restrict__ groups,
             const long long *__restrict__ goff, int n_data, long long row_begin,
             long long row_end, float *__restrict__ ll, long long ll_stride) {
    using G = typename GroupOf<NARROW>::type;
    constexpr int PG = 4;   // groups (16 photons per lane) loaded ahead
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *slf = reinterpret_cast<float *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
    const int gtot = (int)goff[n_data];
    auto lower = [&](int target) {
        int lo = 0, hi = n_data;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)goff[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int fb = wid == 0 ? 0 : lower((int)((long long)gtot * wid / nw));
    const int fe = wid == nw - 1 ? n_data : lower((int)((long long)gtot * (wid + 1) / nw));

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        const float *src = lsl + (first - row_begin) * (long long)p_row;
        stage_tile<T>(slf, src, p_row, nt);
        __syncthreads();
        if (fb >= fe) continue;

        const int my_t = lane & (T - 1);
        const double my_init = my_t < nt ? init[(first + my_t) / num_rot] : 0.;
        float *my_ll = ll + (first + my_t - row_begin) * ll_stride;
        Acc<T> a0, a1;
        a0.zero();
        a1.zero();
        int base = fb;
        int my_end = fb + lane < n_data ? (int)goff[fb + lane + 1] : 0x7fffffff;
        double my_scale = fb + lane < n_data ? scales[fb + lane] : 0.;
        int f = fb;
        int g = (int)goff[fb];
        const int gend = (int)goff[fe];
        int fend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
        auto finish = [&]() {
            Contrib<T> c1;
#pragma unroll
            for (int i = 0; i < (T + 1) / 2; ++i) c1.p[i] = a1.p[i];
            add_contrib<T>(a0, c1);
            const float tot = reduce_scatter<T>(a0, lane);
            const double sc = __shfl_sync(RSPI_FULL_MASK, my_scale, f - base);
            if (lane < nt) my_ll[f] = (float)(my_init * sc + (double)tot);
            a0.zero();
            a1.zero();
            ++f;
            if (f - base == 32) {
                base = f;
                my_end = f + lane < n_data ? (int)goff[f + lane + 1] : 0x7fffffff;
                my_scale = f + lane < n_data ? scales[f + lane] : 0.;
            }
            fend = f < fe ? __shfl_sync(RSPI_FULL_MASK, my_end, f - base) : gend + 1;
        };
        while (f < fe && fend == g) finish();   // frames without entry rows

        const G *gp = groups + (long long)g * 32 + lane;
        G cur[PG], nxt[PG];
        const G z{};
        const unsigned lane_off = 4u * T * (unsigned)(lane % (32 / T));
#pragma unroll
        for (int k = 0; k < PG; ++k) cur[k] = g + k < gend ? __ldg(gp + 32 * k) : z;
        while (g < gend) {
            const int nb = min(PG, gend - g);
#pragma unroll
            for (int k = 0; k < PG; ++k) nxt[k] = g + PG + k < gend ? __ldg(gp + 32 * (PG + k)) : z;
            // gather phase without branches, so the shared loads of all PG
            // groups are in flight together (groups past nb hold offset 0: a
            // valid address whose values are never added)
            Contrib<T> c0[PG], c1[PG];
#pragma unroll
            for (int k = 0; k < PG; ++k) gather_group<T>(smem_raw, cur[k], lane_off, c0[k], c1[k]);
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                if (k < nb) {
                    add_contrib<T>(a0, c0[k]);
                    add_contrib<T>(a1, c1[k]);
                    if (g + k + 1 == fend) {
                        finish();
                        while (f < fe && fend == g + k + 1) finish();
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) cur[k] = nxt[k];
            g += PG;
            gp += 32 * PG;
        }
    }
}

// Frame pairs (two rows per tile, 16-bit entries of k_pair_fill): half-warp
// h of a warp sums frame pair_frames[2 p + h] of pair p, each lane its
// photons of one bank class; a pair's two sums are reduced in one pass of
// four exchange steps inside each half-warp, and lanes 16 h + t store row t
// of frame h.  Warps take contiguous pair ranges of about equal group counts.
__global__ void __launch_bounds__(1024)
k_screen_ll5(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const uint2 *__restrict__ groups, const long long *__restrict__ pgoff,
             const int *__restrict__ pair_frames, int n_pairs, long long row_begin,
             long long row_end, float *__restrict__ ll, long long ll_stride) {
    constexpr int T = 2;
    constexpr int PG = 4;   // groups (4 photons per lane each) loaded ahead
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *slf = reinterpret_cast<float *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int half = lane >> 4, hl = lane & 15;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
    const int gtot = (int)pgoff[n_pairs];
    auto lower = [&](int target) {
        int lo = 0, hi = n_pairs;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)pgoff[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int pb = wid == 0 ? 0 : lower((int)((long long)gtot * wid / nw));
    const int pe = wid == nw - 1 ? n_pairs : lower((int)((long long)gtot * (wid + 1) / nw));
    const unsigned lane_off = 8u * (unsigned)hl;

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        stage_tile<T>(slf, lsl + (first - row_begin) * (long long)p_row, p_row, nt);
        __syncthreads();
        if (pb >= pe) continue;

        const bool storer = hl < nt;   // lanes 16 h + t store row t
        const double my_init = storer ? init[(first + hl) / num_rot] : 0.;
        float *my_ll = ll + (first + (storer ? hl : 0) - row_begin) * ll_stride;
        Acc<T> a0, a1;
        a0.zero();
        a1.zero();
        int base = pb;
        int my_end = pb + lane < n_pairs ? (int)pgoff[pb + lane + 1] : 0x7fffffff;
        int p = pb;
        int g = (int)pgoff[pb];
        const int gend = (int)pgoff[pe];
        int pend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
        // this lane's frame of the current pair and its scale (storers only)
        int my_d = storer ? pair_frames[2 * p + half] : -1;
        double my_sc = my_d >= 0 ? scales[my_d] : 0.;
        auto finish = [&]() {
            float2 a = __fadd2_rn(a0.p[0], a1.p[0]);
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                const float2 b = make_float2(__shfl_xor_sync(RSPI_FULL_MASK, a.x, o),
                                             __shfl_xor_sync(RSPI_FULL_MASK, a.y, o));
                a = __fadd2_rn(a, b);
            }
            if (my_d >= 0) my_ll[my_d] = (float)(my_init * my_sc + (double)(hl == 0 ? a.x : a.y));
            a0.zero();
            a1.zero();
            ++p;
            if (p - base == 32) {
                base = p;
                my_end = p + lane < n_pairs ? (int)pgoff[p + lane + 1] : 0x7fffffff;
            }
            pend = p < pe ? __shfl_sync(RSPI_FULL_MASK, my_end, p - base) : gend + 1;
            my_d = storer && p < pe ? pair_frames[2 * p + half] : -1;
            my_sc = my_d >= 0 ? scales[my_d] : 0.;
        };
        while (p < pe && pend == g) finish();   // pairs without entries

        const uint2 *gp = groups + (long long)g * 32 + lane;
        uint2 cur[PG], nxt[PG];
        const uint2 z{};
#pragma unroll
        for (int k = 0; k < PG; ++k) cur[k] = g + k < gend ? __ldg(gp + 32 * k) : z;
        while (g < gend) {
            const int nb = min(PG, gend - g);
#pragma unroll
            for (int k = 0; k < PG; ++k) nxt[k] = g + PG + k < gend ? __ldg(gp + 32 * (PG + k)) : z;
            Contrib<T> c0[PG], c1[PG];
#pragma unroll
            for (int k = 0; k < PG; ++k) gather_group<T>(smem_raw, cur[k], lane_off, c0[k], c1[k]);
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                if (k < nb) {
                    add_contrib<T>(a0, c0[k]);
                    add_contrib<T>(a1, c1[k]);
                    if (g + k + 1 == pend) {
                        finish();
                        while (p < pe && pend == g + k + 1) finish();
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) cur[k] = nxt[k];
            g += PG;
            gp += 32 * PG;
        }
    }
}

// Frame quads (two rows per tile, 16-bit entries of k_quad_fill): lanes
// 8 u .. 8 u + 7 sum frame quad_frames[4 q + u] of quad q; one pass of three
// exchange steps inside each group of eight lanes reduces all four frames,
// and lanes 8 u + t store row t of frame u.
__global__ void __launch_bounds__(1024)
k_screen_ll6(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const uint2 *__restrict__ groups, const long long *__restrict__ qgoff,
             const int *__restrict__ quad_frames, int n_quads, long long row_begin,
             long long row_end, float *__restrict__ ll, long long ll_stride) {
    constexpr int T = 2;
    constexpr int PG = 4;   // groups (4 photons per lane each) loaded ahead
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *slf = reinterpret_cast<float *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int u = lane >> 3, j = lane & 7;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
    const int gtot = (int)qgoff[n_quads];
    auto lower = [&](int target) {
        int lo = 0, hi = n_quads;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)qgoff[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int qb = wid == 0 ? 0 : lower((int)((long long)gtot * wid / nw));
    const int qe = wid == nw - 1 ? n_quads : lower((int)((long long)gtot * (wid + 1) / nw));
    // byte offsets of the lane's two classes: phase 0 in slots 0, 2, phase 1 in 1, 3
    const unsigned off0 = 8u * (unsigned)(j + 8 * (u & 1));
    const unsigned off1 = 8u * (unsigned)(j + 8 * (1 - (u & 1)));

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        stage_tile<T>(slf, lsl + (first - row_begin) * (long long)p_row, p_row, nt);
        __syncthreads();
        if (qb >= qe) continue;

        const bool storer = j < nt;   // lanes 8 u + t store row t
        const double my_init = storer ? init[(first + j) / num_rot] : 0.;
        float *my_ll = ll + (first + (storer ? j : 0) - row_begin) * ll_stride;
        Acc<T> a0, a1;
        a0.zero();
        a1.zero();
        int base = qb;
        int my_end = qb + lane < n_quads ? (int)qgoff[qb + lane + 1] : 0x7fffffff;
        int q = qb;
        int g = (int)qgoff[qb];
        const int gend = (int)qgoff[qe];
        int qend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
        int my_d = storer ? quad_frames[4 * q + u] : -1;
        double my_sc = my_d >= 0 ? scales[my_d] : 0.;
        auto finish = [&]() {
            float2 a = __fadd2_rn(a0.p[0], a1.p[0]);
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
                const float2 b = make_float2(__shfl_xor_sync(RSPI_FULL_MASK, a.x, o),
                                             __shfl_xor_sync(RSPI_FULL_MASK, a.y, o));
                a = __fadd2_rn(a, b);
            }
            if (my_d >= 0) my_ll[my_d] = (float)(my_init * my_sc + (double)(j == 0 ? a.x : a.y));
            a0.zero();
            a1.zero();
            ++q;
            if (q - base == 32) {
                base = q;
                my_end = q + lane < n_quads ? (int)qgoff[q + lane + 1] : 0x7fffffff;
            }
            qend = q < qe ? __shfl_sync(RSPI_FULL_MASK, my_end, q - base) : gend + 1;
            my_d = storer && q < qe ? quad_frames[4 * q + u] : -1;
            my_sc = my_d >= 0 ? scales[my_d] : 0.;
        };
        while (q < qe && qend == g) finish();   // quads without entries

        const uint2 *gp = groups + (long long)g * 32 + lane;
        uint2 cur[PG], nxt[PG];
        const uint2 z{};
#pragma unroll
        for (int k = 0; k < PG; ++k) cur[k] = g + k < gend ? __ldg(gp + 32 * k) : z;
        while (g < gend) {
            const int nb = min(PG, gend - g);
#pragma unroll
            for (int k = 0; k < PG; ++k) nxt[k] = g + PG + k < gend ? __ldg(gp + 32 * (PG + k)) : z;
            Contrib<T> c0[PG], c1[PG];
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                c0[k] = gather_pair<T>(smem_raw, (cur[k].x & 0xffffu) * 128u + off0,
                                       (cur[k].x >> 16) * 128u + off1);
                c1[k] = gather_pair<T>(smem_raw, (cur[k].y & 0xffffu) * 128u + off0,
                                       (cur[k].y >> 16) * 128u + off1);
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                if (k < nb) {
                    add_contrib<T>(a0, c0[k]);
                    add_contrib<T>(a1, c1[k]);
                    if (g + k + 1 == qend) {
                        finish();
                        while (q < qe && qend == g + k + 1) finish();
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) cur[k] = nxt[k];
            g += PG;
            gp += 32 * PG;
        }
    }
}

// FP16 slices, four rows per tile: the interleaved tile holds sl[c][0..3] as
// halves (8 bytes per pixel), so one 8-byte gather brings four rows' values
// of a photon -- twice the rows per shared-memory wavefront of the FP32
// two-row tile -- and they are widened to FP32 before the packed FP32 adds.
// The wide entries are those of the FP32 two-row tile (offset sel * 8).
__device__ __forceinline__ void gather4h(const unsigned char *sl, unsigned a, unsigned b,
                                         float2 &lo, float2 &hi) {
    const uint2 va = *reinterpret_cast<const uint2 *>(sl + a);
    const uint2 vb = *reinterpret_cast<const uint2 *>(sl + b);
    const float2 a01 = __half22float2(*reinterpret_cast<const __half2 *>(&va.x));
    const float2 a23 = __half22float2(*reinterpret_cast<const __half2 *>(&va.y));
    const float2 b01 = __half22float2(*reinterpret_cast<const __half2 *>(&vb.x));
    const float2 b23 = __half22float2(*reinterpret_cast<const __half2 *>(&vb.y));
    lo = __fadd2_rn(a01, b01);
    hi = __fadd2_rn(a23, b23);
}

__global__ void __launch_bounds__(1024)
k_screen_ll4h(const __half *__restrict__ lsl, int p_row, int num_rot,
              const double *__restrict__ init, const double *__restrict__ scales,
              const uint4 *__restrict__ groups, const long long *__restrict__ goff, int n_data,
              long long row_begin, long long row_end, float *__restrict__ ll,
              long long ll_stride) {
    constexpr int T = 4, PG = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __half *slh = reinterpret_cast<__half *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const long long n_tiles = (row_end - row_begin + T - 1) / T;
    const int gtot = (int)goff[n_data];
    auto lower = [&](int target) {
        int lo = 0, hi = n_data;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)goff[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int fb = wid == 0 ? 0 : lower((int)((long long)gtot * wid / nw));
    const int fe = wid == nw - 1 ? n_data : lower((int)((long long)gtot * (wid + 1) / nw));
    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * T;
        const int nt = (int)min((long long)T, row_end - first);
        __syncthreads();
        const __half *src = lsl + (first - row_begin) * (long long)p_row;
        stage_tile_h<T>(slh, src, p_row, nt);
        __syncthreads();
        if (fb >= fe) continue;

        const int my_t = lane & (T - 1);
        const double my_init = my_t < nt ? init[(first + my_t) / num_rot] : 0.;
        float *my_ll = ll + (first + my_t - row_begin) * ll_stride;
        Acc<T> a0;
        a0.zero();
        int base = fb;
        int my_end = fb + lane < n_data ? (int)goff[fb + lane + 1] : 0x7fffffff;
        double my_scale = fb + lane < n_data ? scales[fb + lane] : 0.;
        int f = fb;
        int g = (int)goff[fb];
        const int gend = (int)goff[fe];
        int fend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
        auto finish = [&]() {
            const float tot = reduce_scatter<T>(a0, lane);
            const double sc = __shfl_sync(RSPI_FULL_MASK, my_scale, f - base);
            if (lane < nt) my_ll[f] = (float)(my_init * sc + (double)tot);
            a0.zero();
            ++f;
            if (f - base == 32) {
                base = f;
                my_end = f + lane < n_data ? (int)goff[f + lane + 1] : 0x7fffffff;
                my_scale = f + lane < n_data ? scales[f + lane] : 0.;
            }
            fend = f < fe ? __shfl_sync(RSPI_FULL_MASK, my_end, f - base) : gend + 1;
        };
        while (f < fe && fend == g) finish();

        const uint4 *gp = groups + (long long)g * 32 + lane;
        uint4 cur[PG], nxt[PG];
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int k = 0; k < PG; ++k) cur[k] = g + k < gend ? __ldg(gp + 32 * k) : z;
        while (g < gend) {
            const int nb = min(PG, gend - g);
#pragma unroll
            for (int k = 0; k < PG; ++k) nxt[k] = g + PG + k < gend ? __ldg(gp + 32 * (PG + k)) : z;
            // a group's four photons summed per row pair before the adds
            Contrib<T> c[PG];
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                float2 l0, h0, l1, h1;
                gather4h(smem_raw, cur[k].x, cur[k].y, l0, h0);
                gather4h(smem_raw, cur[k].z, cur[k].w, l1, h1);
                c[k].p[0] = __fadd2_rn(l0, l1);
                c[k].p[1] = __fadd2_rn(h0, h1);
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) {
                if (k < nb) {
                    add_contrib<T>(a0, c[k]);
                    if (g + k + 1 == fend) {
                        finish();
                        while (f < fe && fend == g + k + 1) finish();
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < PG; ++k) cur[k] = nxt[k];
            g += PG;
            gp += 32 * PG;
        }
    }
}

template <int T, bool NARROW>
int launch4(const float *lsl, long long p_row, long long num_rot, const double *init,
            const double *scales, const typename GroupOf<NARROW>::type *groups,
            const long long *goff, long long n_data, long long r0, long long r1, float *ll,
            long long stride, int warps, int n_ctas, cudaStream_t stream) {
    const size_t smem = (size_t)T * p_row * sizeof(float);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll4<T, NARROW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (r1 - r0 + T - 1) / T;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll4<T, NARROW><<<n_ctas, warps * 32, smem, stream>>>(
        lsl, (int)p_row, (int)num_rot, init, scales, groups, goff, (int)n_data, r0, r1, ll,
        stride);
    RSPI_RETURN_LAUNCH();
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

// Four-row tiles over column parts ("quad4"): four frames per warp as in
// k_screen_ll6, but the tile holds four FP32 rows per column (16 bytes), so
// one 16-byte gather brings all four rows of a photon.  Four FP32 rows of a
// full 185^2 detector row do not fit in shared memory, so the likelihood
// columns [0, p_zero) are cut into n_parts consecutive parts of part_w
// columns (part_w % 8 == 0) plus 8 zero columns, staged one after another.
//
// Entries: lane 8 u + j of a group holds photons of sub-frame u whose local
// column (column - h part_w in part h) is = j (mod 8), four 16-bit q per
// group (local column 8 q + j); the eight lanes of a quarter warp, which one
// 16-byte gather serves per shared-memory wavefront, then touch the eight
// distinct 16-byte bank groups.  The k-th photon of (part h, class j) goes to
// group k / 4, slot k mod 4 of the quad's part-h group range (part-major:
// range h n_quads + q of the offsets); other slots hold q = part_w / 8, the
// zero column part_w + j.  A (quad, part) takes the largest of its frames'
// ceil(max_j n_hj / 4).
constexpr int Q4_MAX_PARTS = 4;

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_quad4_groups(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
               long long n, int p_zero, int n_parts, int part_w, int *__restrict__ groups) {
    __shared__ int cnt[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n; d += nwarp) {
        cnt[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int key = e < (unsigned)p_zero ? (int)(e / (unsigned)part_w) * 8 + (int)(e & 7u)
                                                 : 32;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < 32 && lane == __ffs(m) - 1) cnt[w][key] += __popc(m);
            __syncwarp();
        }
        int mx = cnt[w][lane];
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(RSPI_FULL_MASK, mx, o));
        if ((lane & 7) == 0 && (lane >> 3) < n_parts)
            groups[d * n_parts + (lane >> 3)] = (mx + 3) / 4;
        __syncwarp();
    }
}

__global__ void k_quad4_pad(long long n_slots, unsigned pad_q, uint2 *__restrict__ out) {
    const unsigned pad2 = pad_q | (pad_q << 16);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_slots;
         i += stride)
        out[i] = make_uint2(pad2, pad2);
}

__global__ void __launch_bounds__(BANK_WARPS * 32)
k_quad4_fill(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
             long long n, int p_zero, int n_parts, int part_w, const int *__restrict__ quad_slot,
             const long long *__restrict__ goff, long long n_quads,
             unsigned short *__restrict__ out) {
    __shared__ int base[BANK_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (long long d = warp; d < n; d += nwarp) {
        const int qs = quad_slot[d];
        const long long qd = qs >> 2;
        const int u = qs & 3;
        base[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            const int h = e < (unsigned)p_zero ? (int)(e / (unsigned)part_w) : n_parts;
            const int key = h < n_parts ? h * 8 + (int)(e & 7u) : 32;
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < 32) {
                const int k = base[w][key] + __popc(m & lt);
                const long long gi = (long long)h * n_quads + qd;
                const long long g0 = goff[gi], ng = goff[gi + 1] - g0;
                if ((k >> 2) < ng)
                    out[((g0 + (k >> 2)) * 32 + 8 * u + (key & 7)) * 4 + (k & 3)] =
                        (unsigned short)((e - (unsigned)(h * part_w)) >> 3);
            }
            __syncwarp();
            if (key < 32 && lane == __ffs(m) - 1) base[w][key] += __popc(m);
            __syncwarp();
        }
    }
}

// Part h of four consecutive slice rows into sl4[c] = (row 0..3 at column
// h part_w + c), zeros for rows past nt, columns past p_row and the 8 pad
// columns part_w .. part_w + 7.
__device__ __forceinline__ void stage_part4(float4 *sl4, const float *__restrict__ src, int p_row,
                                            int nt, int c0, int part_w) {
    const int width = part_w + 8;
#pragma unroll 4
    for (int c = threadIdx.x; c < width; c += blockDim.x) {
        const int gc = c0 + c;
        const bool in = c < part_w && gc < p_row;
        float v[4];
#pragma unroll
        for (int t = 0; t < 4; ++t)
            v[t] = in && t < nt ? __ldg(src + (long long)t * p_row + gc) : 0.f;
        sl4[c] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// One 16-byte gather per photon: photon a's four rows + photon b's.
__device__ __forceinline__ Contrib<4> gather_pair4(const unsigned char *sl, unsigned a,
                                                   unsigned b) {
    const float4 va = *reinterpret_cast<const float4 *>(sl + a);
    const float4 vb = *reinterpret_cast<const float4 *>(sl + b);
    Contrib<4> c;
    c.p[0] = __fadd2_rn(make_float2(va.x, va.y), make_float2(vb.x, vb.y));
    c.p[1] = __fadd2_rn(make_float2(va.z, va.w), make_float2(vb.z, vb.w));
    return c;
}

// Lanes 8 u + j sum frame quad_frames[4 q + u] of quad q over the part's
// groups; after three exchange steps (xor 4: row pair, xor 2: row, xor 1)
// lanes 8 u + 2 t and 8 u + 2 t + 1 hold row t's sum and lane 8 u + 2 t
// stores it.  With several parts the running sum of (row t, slot 4 q + u)
// is kept in part_sums[cta][t][4 q + u] (parts before the last) and added
// in FP64 to the last part's sum before the final FP32 rounding.  Warps take
// contiguous quad ranges of about equal groups over all parts.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
k_screen_ll7(const float *__restrict__ lsl, int p_row, int num_rot,
             const double *__restrict__ init, const double *__restrict__ scales,
             const uint2 *__restrict__ groups, const long long *__restrict__ goff,
             const int *__restrict__ quad_frames, int n_quads, int n_parts, int part_w,
             long long row_begin, long long row_end, float *__restrict__ ll, long long ll_stride,
             float *part_sums) {
    constexpr int PG = 2;   // groups (4 photons per lane each) loaded ahead
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4 *sl4 = reinterpret_cast<float4 *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int u = lane >> 3, j = lane & 7;
    const long long n_tiles = (row_end - row_begin + 3) / 4;
    auto comb = [&](int q) {
        long long s = 0;
        for (int h = 0; h < n_parts; ++h)
            s += goff[(long long)h * n_quads + q] - goff[(long long)h * n_quads];
        return s;
    };
    const long long gtot = comb(n_quads);
    auto lower = [&](long long target) {
        int lo = 0, hi = n_quads;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (comb(mid) < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const int qb = wid == 0 ? 0 : lower(gtot * wid / nw);
    const int qe = wid == nw - 1 ? n_quads : lower(gtot * (wid + 1) / nw);
    const unsigned lane_off = 16u * (unsigned)j;
    const int t_st = j >> 1;
    float *my_ps = part_sums ? part_sums + ((long long)blockIdx.x * 4 + t_st) * (4LL * n_quads) + u
                             : nullptr;

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long long first = row_begin + tile * 4;
        const int nt = (int)min(4LL, row_end - first);
        const bool storer = (j & 1) == 0 && t_st < nt;
        const double my_init = storer ? init[(first + t_st) / num_rot] : 0.;
        float *my_ll = ll + (first + (storer ? t_st : 0) - row_begin) * ll_stride;
        for (int h = 0; h < n_parts; ++h) {
            __syncthreads();
            stage_part4(sl4, lsl + (first - row_begin) * (long long)p_row, p_row, nt,
                        h * part_w, part_w);
            __syncthreads();
            if (qb >= qe) continue;
            const bool last = h == n_parts - 1, firstp = h == 0;
            const long long *go = goff + (long long)h * n_quads;
            Acc<4> a0, a1;
            a0.zero();
            a1.zero();
            int base = qb;
            int my_end = qb + lane < n_quads ? (int)go[qb + lane + 1] : 0x7fffffff;
            int q = qb;
            int g = (int)go[qb];
            const int gend = (int)go[qe];
            int qend = __shfl_sync(RSPI_FULL_MASK, my_end, 0);
            int my_d = storer && last ? quad_frames[4 * q + u] : -1;
            double my_sc = my_d >= 0 ? scales[my_d] : 0.;
            float my_prev = storer && !firstp ? my_ps[4LL * q] : 0.f;
            auto finish = [&]() {
                float2 p0 = __fadd2_rn(a0.p[0], a1.p[0]);
                float2 p1 = __fadd2_rn(a0.p[1], a1.p[1]);
                // xor 4: keep the row pair (j >> 2) & 1
                const bool b2 = j & 4;
                float2 keep = b2 ? p1 : p0;
                const float2 send = b2 ? p0 : p1;
                keep = __fadd2_rn(keep, make_float2(__shfl_xor_sync(RSPI_FULL_MASK, send.x, 4),
                                                    __shfl_xor_sync(RSPI_FULL_MASK, send.y, 4)));
                // xor 2: keep row (j >> 1) & 1 of the pair
                const bool b1 = j & 2;
                float s = b1 ? keep.y : keep.x;
                s += __shfl_xor_sync(RSPI_FULL_MASK, b1 ? keep.x : keep.y, 2);
                s += __shfl_xor_sync(RSPI_FULL_MASK, s, 1);
                if (storer) {
                    if (last) {
                        if (my_d >= 0)
                            my_ll[my_d] = (float)(my_init * my_sc + ((double)my_prev + (double)s));
                    } else {
                        my_ps[4LL * q] = firstp ? s : (float)((double)my_prev + (double)s);
                    }
                }
                a0.zero();
                a1.zero();
                ++q;
                if (q - base == 32) {
                    base = q;
                    my_end = q + lane < n_quads ? (int)go[q + lane + 1] : 0x7fffffff;
                }
                qend = q < qe ? __shfl_sync(RSPI_FULL_MASK, my_end, q - base) : gend + 1;
                my_d = storer && last && q < qe ? quad_frames[4 * q + u] : -1;
                my_sc = my_d >= 0 ? scales[my_d] : 0.;
                my_prev = storer && !firstp && q < qe ? my_ps[4LL * q] : 0.f;
            };
            while (q < qe && qend == g) finish();   // quads without entries in this part

            const uint2 *gp = groups + (long long)g * 32 + lane;
            uint2 cur[PG], nxt[PG];
            const uint2 z{};
#pragma unroll
            for (int k = 0; k < PG; ++k) cur[k] = g + k < gend ? __ldg(gp + 32 * k) : z;
            while (g < gend) {
                const int nb = min(PG, gend - g);
#pragma unroll
                for (int k = 0; k < PG; ++k)
                    nxt[k] = g + PG + k < gend ? __ldg(gp + 32 * (PG + k)) : z;
                Contrib<4> c0[PG], c1[PG];
#pragma unroll
                for (int k = 0; k < PG; ++k) {
                    c0[k] = gather_pair4(smem_raw, (cur[k].x & 0xffffu) * 128u + lane_off,
                                         (cur[k].x >> 16) * 128u + lane_off);
                    c1[k] = gather_pair4(smem_raw, (cur[k].y & 0xffffu) * 128u + lane_off,
                                         (cur[k].y >> 16) * 128u + lane_off);
                }
#pragma unroll
                for (int k = 0; k < PG; ++k) {
                    if (k < nb) {
                        add_contrib<4>(a0, c0[k]);
                        add_contrib<4>(a1, c1[k]);
                        if (g + k + 1 == qend) {
                            finish();
                            while (q < qe && qend == g + k + 1) finish();
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < PG; ++k) cur[k] = nxt[k];
                g += PG;
                gp += 32 * PG;
            }
        }
    }
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

extern "C" int rspi_screen_loglike3(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned short *entries, const long long *row_off,
                                    long long n_data, long long row_begin, long long row_end,
                                    float *ll, long long ll_stride, int states_per_tile,
                                    int prefetch_words, int warps_per_cta, int n_ctas,
                                    cudaStream_t stream) {
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
#define RSPI_LL3(T, PF)                                                                        \
    return launch3<T, PF>(lslices, p_row, num_rot, init, scales, w, row_off, n_data, row_begin, \
                          row_end, ll, ll_stride, warps_per_cta, n_ctas, stream)
    if (states_per_tile == 1) {
        if (prefetch_words == 4) RSPI_LL3(1, 4);
        if (prefetch_words == 8) RSPI_LL3(1, 8);
        if (prefetch_words == 12) RSPI_LL3(1, 12);
    } else if (states_per_tile == 2) {
        if (prefetch_words == 4) RSPI_LL3(2, 4);
        if (prefetch_words == 8) RSPI_LL3(2, 8);
        if (prefetch_words == 12) RSPI_LL3(2, 12);
    }
#undef RSPI_LL3
    return RSPI_ERR_ARG;
}

extern "C" int rspi_wide_entry_groups(const long long *row_off16, long long n_data, int *groups,
                                      cudaStream_t stream) {
    if (!row_off16 || !groups || n_data <= 0) return RSPI_ERR_ARG;
    k_wide_groups<<<rspi_blocks(n_data, 256), 256, 0, stream>>>(row_off16, n_data, groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_wide_entry_fill(const unsigned short *entries16, const long long *row_off16,
                                    long long n_data, int p_zero, int states_per_tile,
                                    const long long *group_off, unsigned *wide,
                                    cudaStream_t stream) {
    if (!entries16 || !row_off16 || !group_off || !wide || n_data <= 0 || p_zero < 0 ||
        p_zero % 32 || p_zero + 32 > 65536 || (states_per_tile != 1 && states_per_tile != 2))
        return RSPI_ERR_ARG;
    k_wide_fill<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, states_per_tile, group_off, wide);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_wide_entry_groups_banked(const unsigned short *entries16,
                                             const long long *row_off16, long long n_data,
                                             int p_zero, int states_per_tile, int *groups,
                                             cudaStream_t stream) {
    if (!entries16 || !row_off16 || !groups || n_data <= 0 || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536 || (states_per_tile != 1 && states_per_tile != 2))
        return RSPI_ERR_ARG;
    k_wide_groups_banked<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0,
                           stream>>>(entries16, row_off16, n_data, p_zero, 32 / states_per_tile,
                                     4 * states_per_tile, groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_wide_entry_fill_banked(const unsigned short *entries16,
                                           const long long *row_off16, long long n_data,
                                           int p_zero, int states_per_tile,
                                           const long long *group_off, unsigned *wide,
                                           cudaStream_t stream) {
    if (!entries16 || !row_off16 || !group_off || !wide || n_data <= 0 || p_zero < 0 ||
        p_zero % 32 || p_zero + 32 > 65536 || (states_per_tile != 1 && states_per_tile != 2))
        return RSPI_ERR_ARG;
    k_wide_fill_banked<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0,
                         stream>>>(entries16, row_off16, n_data, p_zero, 32 / states_per_tile,
                                   4u * (unsigned)states_per_tile, group_off, wide);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_wide_entry_fill_narrow(const unsigned short *entries16,
                                           const long long *row_off16, long long n_data,
                                           int p_zero, int states_per_tile,
                                           const long long *group_off, unsigned short *narrow,
                                           cudaStream_t stream) {
    if (!entries16 || !row_off16 || !group_off || !narrow || n_data <= 0 || p_zero < 0 ||
        p_zero % 32 || p_zero + 32 > 65536 || (states_per_tile != 1 && states_per_tile != 2) ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    k_narrow_fill_banked<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0,
                           stream>>>(entries16, row_off16, n_data, p_zero, 32 / states_per_tile,
                                     group_off, narrow);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_screen_loglike4(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned *wide, const long long *group_off,
                                    long long n_data, long long row_begin, long long row_end,
                                    float *ll, long long ll_stride, int states_per_tile,
                                    int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !wide || !group_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin || ll_stride < n_data ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(wide) & 15) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const uint4 *g = reinterpret_cast<const uint4 *>(wide);
    if (states_per_tile == 1)
        return launch4<1, false>(lslices, p_row, num_rot, init, scales, g, group_off, n_data,
                                 row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    if (states_per_tile == 2)
        return launch4<2, false>(lslices, p_row, num_rot, init, scales, g, group_off, n_data,
                                 row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    return RSPI_ERR_ARG;
}

extern "C" int rspi_screen_loglike4n(const float *lslices, long long p_row, long long num_rot,
                                     const double *init, const double *scales,
                                     const unsigned short *narrow, const long long *group_off,
                                     long long n_data, long long row_begin, long long row_end,
                                     float *ll, long long ll_stride, int states_per_tile,
                                     int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !narrow || !group_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin || ll_stride < n_data ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const uint2 *g = reinterpret_cast<const uint2 *>(narrow);
    if (states_per_tile == 1)
        return launch4<1, true>(lslices, p_row, num_rot, init, scales, g, group_off, n_data,
                                row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    if (states_per_tile == 2)
        return launch4<2, true>(lslices, p_row, num_rot, init, scales, g, group_off, n_data,
                                row_begin, row_end, ll, ll_stride, warps_per_cta, n_ctas, stream);
    return RSPI_ERR_ARG;
}

extern "C" int rspi_screen_loglike4h(const void *lslices16, long long p_row, long long num_rot,
                                     const double *init, const double *scales,
                                     const unsigned *wide, const long long *group_off,
                                     long long n_data, long long row_begin, long long row_end,
                                     float *ll, long long ll_stride, int warps_per_cta,
                                     int n_ctas, cudaStream_t stream) {
    if (!lslices16 || !init || !scales || !wide || !group_off || !ll || n_data <= 0 ||
        n_data > 0x7fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin || ll_stride < n_data ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices16) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(wide) & 15) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const size_t smem = (size_t)4 * p_row * sizeof(__half);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll4h, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (row_end - row_begin + 3) / 4;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps_per_cta * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll4h<<<n_ctas, warps_per_cta * 32, smem, stream>>>(
        (const __half *)lslices16, (int)p_row, (int)num_rot, init, scales,
        reinterpret_cast<const uint4 *>(wide), group_off, (int)n_data, row_begin, row_end, ll,
        ll_stride);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_pair_entry_groups(const unsigned short *entries16, const long long *row_off16,
                                      long long n_data, int p_zero, int *groups,
                                      cudaStream_t stream) {
    if (!entries16 || !row_off16 || !groups || n_data <= 0 || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536)
        return RSPI_ERR_ARG;
    k_wide_groups_banked<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0,
                           stream>>>(entries16, row_off16, n_data, p_zero, 16, 4, groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_pair_entry_fill(const unsigned short *entries16, const long long *row_off16,
                                    long long n_data, int p_zero, const int *pair_slot,
                                    const long long *pair_group_off, long long total_groups,
                                    unsigned short *narrow, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !pair_slot || !pair_group_off || !narrow || n_data <= 0 ||
        p_zero < 0 || p_zero % 32 || p_zero + 32 > 65536 || total_groups < 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (total_groups > 0)
        k_pair_pad<<<rspi_blocks(total_groups * 32, 256), 256, 0, stream>>>(
            total_groups * 32, p_zero, reinterpret_cast<uint2 *>(narrow));
    k_pair_fill<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, pair_slot, pair_group_off, narrow);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_screen_loglike5(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned short *narrow, const long long *pair_group_off,
                                    const int *pair_frames, long long n_pairs, long long row_begin,
                                    long long row_end, float *ll, long long ll_stride,
                                    int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !narrow || !pair_group_off || !pair_frames || !ll ||
        n_pairs <= 0 || n_pairs > 0x3fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 ||
        num_rot <= 0 || num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const size_t smem = 2 * (size_t)p_row * sizeof(float);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll5, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (row_end - row_begin + 1) / 2;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps_per_cta * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll5<<<n_ctas, warps_per_cta * 32, smem, stream>>>(
        lslices, (int)p_row, (int)num_rot, init, scales, reinterpret_cast<const uint2 *>(narrow),
        pair_group_off, pair_frames, (int)n_pairs, row_begin, row_end, ll, ll_stride);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_quad_entry_groups(const unsigned short *entries16, const long long *row_off16,
                                      long long n_data, int p_zero, int *groups,
                                      cudaStream_t stream) {
    if (!entries16 || !row_off16 || !groups || n_data <= 0 || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536)
        return RSPI_ERR_ARG;
    k_wide_groups_banked<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0,
                           stream>>>(entries16, row_off16, n_data, p_zero, 16, 2, groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_quad_entry_fill(const unsigned short *entries16, const long long *row_off16,
                                    long long n_data, int p_zero, const int *quad_slot,
                                    const long long *quad_group_off, long long total_groups,
                                    unsigned short *narrow, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !quad_slot || !quad_group_off || !narrow || n_data <= 0 ||
        p_zero < 0 || p_zero % 32 || p_zero + 32 > 65536 || total_groups < 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (total_groups > 0)
        k_quad_pad<<<rspi_blocks(total_groups * 32, 256), 256, 0, stream>>>(
            total_groups * 32, p_zero, reinterpret_cast<uint2 *>(narrow));
    k_quad_fill<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, quad_slot, quad_group_off, narrow);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_screen_loglike6(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned short *narrow, const long long *quad_group_off,
                                    const int *quad_frames, long long n_quads, long long row_begin,
                                    long long row_end, float *ll, long long ll_stride,
                                    int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !narrow || !quad_group_off || !quad_frames || !ll ||
        n_quads <= 0 || n_quads > 0x1fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 ||
        num_rot <= 0 || num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin ||
        warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const size_t smem = 2 * (size_t)p_row * sizeof(float);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(k_screen_ll6, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RSPI_ERR_CUDA;
        smem_set = smem;
    }
    const long long n_tiles = (row_end - row_begin + 1) / 2;
    if (n_ctas <= 0) {
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps_per_cta * 32)));
    }
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    k_screen_ll6<<<n_ctas, warps_per_cta * 32, smem, stream>>>(
        lslices, (int)p_row, (int)num_rot, init, scales, reinterpret_cast<const uint2 *>(narrow),
        quad_group_off, quad_frames, (int)n_quads, row_begin, row_end, ll, ll_stride);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_quad4_entry_groups(const unsigned short *entries16, const long long *row_off16,
                                       long long n_data, int p_zero, int n_parts, int part_w,
                                       int *groups, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !groups || n_data <= 0 || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536 || n_parts < 1 || n_parts > Q4_MAX_PARTS || part_w < 8 ||
        part_w % 8 || (long long)n_parts * part_w < p_zero)
        return RSPI_ERR_ARG;
    k_quad4_groups<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, n_parts, part_w, groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_quad4_entry_fill(const unsigned short *entries16, const long long *row_off16,
                                     long long n_data, int p_zero, int n_parts, int part_w,
                                     const int *quad_slot, const long long *group_off,
                                     long long n_quads, long long total_groups,
                                     unsigned short *narrow, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !quad_slot || !group_off || !narrow || n_data <= 0 ||
        p_zero < 0 || p_zero % 32 || p_zero + 32 > 65536 || n_parts < 1 ||
        n_parts > Q4_MAX_PARTS || part_w < 8 || part_w % 8 ||
        (long long)n_parts * part_w < p_zero || part_w / 8 > 0xffff || n_quads <= 0 ||
        n_quads * 4 < n_data || total_groups < 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (total_groups > 0)
        k_quad4_pad<<<rspi_blocks(total_groups * 32, 256), 256, 0, stream>>>(
            total_groups * 32, (unsigned)(part_w / 8), reinterpret_cast<uint2 *>(narrow));
    k_quad4_fill<<<rspi_blocks(n_data * 32, BANK_WARPS * 32), BANK_WARPS * 32, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, n_parts, part_w, quad_slot, group_off, n_quads,
        narrow);
    RSPI_RETURN_LAUNCH();
}

extern "C" long long rspi_quad4_part_sums_floats(long long n_quads, int n_ctas) {
    if (n_quads <= 0 || n_ctas <= 0) return -1;
    return (long long)n_ctas * 16LL * n_quads;
}

extern "C" int rspi_screen_loglike7(const float *lslices, long long p_row, long long num_rot,
                                    const double *init, const double *scales,
                                    const unsigned short *narrow, const long long *group_off,
                                    const int *quad_frames, long long n_quads, int n_parts,
                                    int part_w, long long row_begin, long long row_end, float *ll,
                                    long long ll_stride, float *part_sums, int part_sums_ctas,
                                    int warps_per_cta, int n_ctas, cudaStream_t stream) {
    if (!lslices || !init || !scales || !narrow || !group_off || !quad_frames || !ll ||
        n_quads <= 0 || n_quads > 0x1fffffffLL || p_row <= 32 || p_row % 32 || p_row > 65536 ||
        num_rot <= 0 || num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin ||
        n_parts < 1 || n_parts > Q4_MAX_PARTS || part_w < 8 || part_w % 8 ||
        (long long)n_parts * part_w < p_row - 32 || warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    if (n_parts > 1 && (!part_sums || part_sums_ctas < 1)) return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(narrow) & 7) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const size_t smem = (size_t)(part_w + 8) * sizeof(float4);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    const long long n_tiles = (row_end - row_begin + 3) / 4;
    const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
    if (n_ctas <= 0) n_ctas = rspi_sm_count() * min(per_sm, max(1, 2048 / (warps_per_cta * 32)));
    if (n_parts > 1 && n_ctas > part_sums_ctas) n_ctas = part_sums_ctas;
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    float *ps = n_parts > 1 ? part_sums : nullptr;
    if (warps_per_cta <= 24) {
        static size_t smem_set = 0;
        if (smem > smem_set) {
            if (cudaFuncSetAttribute(k_screen_ll7<768>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem) != cudaSuccess)
                return RSPI_ERR_CUDA;
            smem_set = smem;
        }
        k_screen_ll7<768><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            lslices, (int)p_row, (int)num_rot, init, scales,
            reinterpret_cast<const uint2 *>(narrow), group_off, quad_frames, (int)n_quads,
            n_parts, part_w, row_begin, row_end, ll, ll_stride, ps);
    } else {
        static size_t smem_set = 0;
        if (smem > smem_set) {
            if (cudaFuncSetAttribute(k_screen_ll7<1024>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem) != cudaSuccess)
                return RSPI_ERR_CUDA;
            smem_set = smem;
        }
        k_screen_ll7<1024><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            lslices, (int)p_row, (int)num_rot, init, scales,
            reinterpret_cast<const uint2 *>(narrow), group_off, quad_frames, (int)n_quads,
            n_parts, part_w, row_begin, row_end, ll, ll_stride, ps);
    }
    RSPI_RETURN_LAUNCH();
}
