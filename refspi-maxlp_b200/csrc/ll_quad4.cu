// Screening likelihood, four-row frame-quad form (row a7, the FP32
// screening pass of the chosen form).
//
// The FP32 slices of four consecutive likelihood rows are staged in shared
// memory interleaved by column, sl4[c] = (row 0..3 at column c), so one
// 16-byte gather brings a photon's value in all four rows.  Four FP32 rows
// of a 185^2 detector's likelihood columns do not fit in shared memory, so
// the columns are cut into parts staged one after another.  The photon
// entries come from the 16-bit layout of rspi_ll16_entry_fill, validated
// once on the host side of the pipeline (rspi_entries16_check), so the hot
// loop has no clamp.
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;

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
__device__ __forceinline__ void add_contrib(Acc<T> &a, const Contrib<T> &c) {
    if (T == 1) {
        a.p[0].x += c.p[0].x;
    } else {
#pragma unroll
        for (int i = 0; i < (T + 1) / 2; ++i) a.p[i] = __fadd2_rn(a.p[i], c.p[i]);
    }
}

constexpr int BANK_WARPS = 8;

// Entry r of lane `lane` in the 16-bit entry rows (two rows per 32-bit word).
__device__ __forceinline__ unsigned entry16_at(const unsigned short *__restrict__ ent16,
                                               long long rr, int lane) {
    return ent16[(rr >> 1) * 64 + lane * 2 + (rr & 1)];
}

// Four-row tiles over column parts ("quad4"): four frames per warp, eight
// lanes each; the tile holds four FP32 rows per column (16 bytes), so one
// 16-byte gather brings all four rows of a photon.  Four FP32 rows of a
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
        static RspiSmemOptIn optin;
        if (!rspi_smem_optin((const void *)k_screen_ll7<768>, smem, optin)) return RSPI_ERR_CUDA;
        k_screen_ll7<768><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            lslices, (int)p_row, (int)num_rot, init, scales,
            reinterpret_cast<const uint2 *>(narrow), group_off, quad_frames, (int)n_quads,
            n_parts, part_w, row_begin, row_end, ll, ll_stride, ps);
    } else {
        static RspiSmemOptIn optin;
        if (!rspi_smem_optin((const void *)k_screen_ll7<1024>, smem, optin)) return RSPI_ERR_CUDA;
        k_screen_ll7<1024><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            lslices, (int)p_row, (int)num_rot, init, scales,
            reinterpret_cast<const uint2 *>(narrow), group_off, quad_frames, (int)n_quads,
            n_parts, part_w, row_begin, row_end, ll, ll_stride, ps);
    }
    RSPI_RETURN_LAUNCH();
}
