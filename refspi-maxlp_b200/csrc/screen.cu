// Screened likelihood (rows a7-a9, the chosen form).
//
// 1. FP32 screening pass (ll_sets.cu, ll_quad4.cu, ll_stream.cu): rotated
//    log-slices stored in FP32, photons as 16-bit sel indices with counts
//    expanded (a pixel with k photons is k entries, built here).  Sums are
//    FP32.
// 2. Per frame, every state whose screened value is within
//    delta + 2 * eps_d of the frame's screened maximum becomes a candidate,
//    where eps_d bounds |LL32 - LL64| (storage rounding of the slices,
//    FP32 summation, output rounding).  Any state that is the FP64 argmax or
//    carries posterior mass above exp(-delta) is a candidate.
// 3. Candidates are rescored in FP64 with the same slice function, packed
//    entries and summation order as the FP64 form, so rmax, the maximum and
//    the log-sum-exp equal the FP64 form's values.
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;
constexpr int ENTRY_WARPS = 8;
constexpr double U32 = 5.9604644775390625e-08;  // 2^-24, FP32 unit roundoff

// ---------------------------------------------------------------------------
// 16-bit count-expanded entry lists
// ---------------------------------------------------------------------------
struct Ent {
    int c;    // sel index or -1
    int cnt;  // photons
};

__device__ __forceinline__ Ent entry_at(int i, int n_o, long long oa, long long ma,
                                        const int *place_ones, const int *place_multi,
                                        const int *count_multi, const int *pix2sel,
                                        long long num_pix) {
    Ent e{-1, 0};
    int p;
    if (i < n_o) {
        p = place_ones[oa + i];
        e.cnt = 1;
    } else {
        p = place_multi[ma + (i - n_o)];
        e.cnt = count_multi[ma + (i - n_o)];
    }
    if (p < 0 || p >= num_pix || e.cnt <= 0) return e;
    e.c = pix2sel[p];
    return e;
}

// rows per frame = largest bank population counting copies, rounded up to even
__global__ void __launch_bounds__(ENTRY_WARPS * 32)
k_entry16_rows(const int *__restrict__ ones, const int *__restrict__ multi,
               const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
               const int *__restrict__ place_ones, const int *__restrict__ place_multi,
               const int *__restrict__ count_multi, const int *__restrict__ pix2sel,
               long long num_pix, long long n, int p_zero, int *__restrict__ frame_rows,
               int *err) {
    __shared__ int hist[ENTRY_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long nwarp = (long long)gridDim.x * ENTRY_WARPS;
    for (long long d = (long long)blockIdx.x * ENTRY_WARPS + w; d < n; d += nwarp) {
        hist[w][lane] = 0;
        __syncwarp();
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
        for (int i = lane; i < n_o + n_m; i += 32) {
            Ent e = entry_at(i, n_o, oa, ma, place_ones, place_multi, count_multi, pix2sel,
                             num_pix);
            if (e.c >= 0) {
                if (e.c >= p_zero) rspi_flag(err, RSPI_ERR_CAPACITY);
                else atomicAdd(&hist[w][e.c & 31], e.cnt);
            }
        }
        __syncwarp();
        int rows = warp_max_int(hist[w][lane]);
        if (lane == 0) frame_rows[d] = (rows + 1) & ~1;
        __syncwarp();
    }
}

// Deterministic fill: a lane's copies occupy consecutive slots of its bank,
// after the copies of same-bank entries of lower lanes in the same chunk.
// Layout: word (pair, lane) holds rows 2*pair (low half) and 2*pair+1.
__global__ void __launch_bounds__(ENTRY_WARPS * 32)
k_entry16_fill(const int *__restrict__ ones, const int *__restrict__ multi,
               const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
               const int *__restrict__ place_ones, const int *__restrict__ place_multi,
               const int *__restrict__ count_multi, const int *__restrict__ pix2sel,
               long long num_pix, long long n, int p_zero, const long long *__restrict__ row_off,
               unsigned short *__restrict__ ent) {
    __shared__ int base[ENTRY_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long nwarp = (long long)gridDim.x * ENTRY_WARPS;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (long long d = (long long)blockIdx.x * ENTRY_WARPS + w; d < n; d += nwarp) {
        base[w][lane] = 0;
        __syncwarp();
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
        const long long r0 = row_off[d], nrows = row_off[d + 1] - r0;
        for (int i0 = 0; i0 < n_o + n_m; i0 += 32) {
            const int i = i0 + lane;
            Ent e{-1, 0};
            if (i < n_o + n_m)
                e = entry_at(i, n_o, oa, ma, place_ones, place_multi, count_multi, pix2sel,
                             num_pix);
            if (e.c >= p_zero) e.c = -1;
            const int key = e.c >= 0 ? (e.c & 31) : 32 + lane;
            const unsigned peers = __match_any_sync(RSPI_FULL_MASK, key);
            // copies of lower same-bank lanes come first
            int before = 0, total = 0;
            unsigned m = peers;
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const int c = __shfl_sync(peers, e.cnt, l);
                if (l < lane) before += c;
                total += c;
            }
            if (e.c >= 0) {
                const int b = e.c & 31;
                const long long s0 = base[w][b] + before;
                for (int k = 0; k < e.cnt; ++k) {
                    const long long r = s0 + k;
                    if (r < nrows) {
                        const long long rr = r0 + r;
                        ent[(rr >> 1) * 64 + b * 2 + (rr & 1)] = (unsigned short)e.c;
                    }
                }
            }
            __syncwarp();
            if (e.c >= 0 && (peers & lt_mask) == 0) base[w][e.c & 31] += total;
            __syncwarp();
        }
        for (long long r = base[w][lane]; r < nrows; ++r) {
            const long long rr = r0 + r;
            ent[(rr >> 1) * 64 + lane * 2 + (rr & 1)] = (unsigned short)(p_zero + lane);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// candidate selection
// ---------------------------------------------------------------------------
constexpr int RY = 32;

__device__ __forceinline__ double frame_eps(long long phot, long long rows, float lmax,
                                            double maxll, double delta) {
    // slice rounding + FP32 summation (per-lane sequential + 5-level tree)
    // + output rounding, for every state within delta of the maximum
    const double sum_abs = (double)phot * (double)lmax;
    return U32 * ((double)(rows + 8) * sum_abs + fabs(maxll) + delta + 1.) + 1e-9 * sum_abs;
}

// cnt_part[d * RY + t]: thread t's candidate count of frame d, with its
// second candidate's row when it has two: low 2 bits min(count, 3), above
// them the count (3 or more) or the second row's step k (row t + RY k).
__device__ __forceinline__ int cnt_pack(int c, int k2) {
    return c <= 2 ? (c | (k2 << 2)) : (3 | (c << 2));
}
__device__ __forceinline__ int cnt_count(int v) { return (v & 3) < 3 ? (v & 3) : (v >> 2); }

__global__ void __launch_bounds__(32 * RY)
k_cand_count(const float *__restrict__ ll, long long n_rows, long long n_x, long long stride,
             const int *__restrict__ frame_of_col,
             const double *__restrict__ max32, const int *__restrict__ rmax32,
             const long long *__restrict__ phot,
             const long long *__restrict__ row_off16, const float *__restrict__ lmax, double delta,
             int *__restrict__ cnt_part /* n_data x RY */, int *__restrict__ cand_n,
             double *__restrict__ noncand, double *__restrict__ thr_out,
             int *__restrict__ cand_slot /* n_data x RY, or null */) {
    __shared__ int sc[RY][33];
    __shared__ double sn[RY][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    // thread column x of the likelihood matrix holds frame d (x itself
    // unless the columns are a permutation of the frames)
    const long long x = (long long)blockIdx.x * 32 + tx;
    const long long d = x >= n_x ? -1 : (frame_of_col ? (long long)frame_of_col[x] : x);
    int c = 0, first = -1, second = 0;
    double nc = 0.;
    if (d >= 0) {
        const double m = max32[d];
        const long long rows = row_off16[d + 1] - row_off16[d];
        const double thr = m - delta - 2. * frame_eps(phot[d], rows, *lmax, m, delta);
        const int rm = rmax32[d];
        // FP32 forms of the test and the term, the same decisions and bits:
        // v >= thr32 exactly when (double)v >= thr (thr32 the least float
        // not below thr), and m is a float value (the FP32 matrix's
        // maximum), so v - m in FP32 is the double difference rounded to
        // float whenever exp of it is not zero
        float thr32 = (float)thr;
        if ((double)thr32 < thr) thr32 = nextafterf(thr32, INFINITY);
        const float m32 = (float)m;
        auto take = [&](float v, long long rr) {
            if (v >= thr32 || rr == rm) {
                if (c == 0) first = (int)rr;
                else if (c == 1) second = (int)rr;
                ++c;
            } else {
                nc += (double)expf(v - m32);   // each term < exp(-delta)
            }
        };
        // eight rows' loads in flight per thread, taken in row order
        long long r = ty;
        for (; r + 7 * RY < n_rows; r += 8 * RY) {
            float v8[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v8[u] = __ldg(&ll[(r + u * RY) * stride + x]);
#pragma unroll
            for (int u = 0; u < 8; ++u) take(v8[u], r + u * RY);
        }
        for (; r < n_rows; r += RY) take(ll[r * stride + x], r);
        cnt_part[d * RY + ty] = cnt_pack(c, c == 2 ? (second - ty) / RY : 0);
        // the thread's first candidate row when it has one or two (-2: more)
        if (cand_slot) cand_slot[d * RY + ty] = c > 2 ? -2 : first;
        if (ty == 0) thr_out[d] = thr;
    }
    sc[ty][tx] = c;
    sn[ty][tx] = nc;
    __syncthreads();
    if (ty == 0 && d >= 0) {
        int tot = 0;
        double s = 0.;
        for (int k = 0; k < RY; ++k) {
            tot += sc[k][tx];
            s += sn[k][tx];
        }
        cand_n[d] = tot;
        noncand[d] = s;
    }
}

__global__ void __launch_bounds__(32 * RY)
k_cand_fill(const float *__restrict__ ll, long long n_rows, long long n_x, long long stride,
            const int *__restrict__ frame_of_col, const int *__restrict__ cand_slot,
            const double *__restrict__ thr, const int *__restrict__ rmax32,
            const int *__restrict__ cnt_part,
            const long long *__restrict__ cand_off, long long capacity,
            int *__restrict__ cand_d, int *__restrict__ cand_r, int *err) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long x = (long long)blockIdx.x * 32 + tx;
    const long long d = x >= n_x ? -1 : (frame_of_col ? (long long)frame_of_col[x] : x);
    if (cand_slot) {
        // only frames in which some thread had three or more candidates
        // are filled here (k_cand_compact took the others)
        __shared__ int over[32];
        if (ty == 0) over[tx] = 0;
        __syncthreads();
        if (d >= 0 && cand_slot[d * RY + ty] == -2) over[tx] = 1;
        __syncthreads();
        if (!over[tx]) return;
    }
    if (d < 0) return;
    long long pos = cand_off[d];
    for (int k = 0; k < ty; ++k) pos += cnt_count(cnt_part[d * RY + k]);
    const double th = thr[d];
    const int rm = rmax32[d];
    auto take = [&](float v, long long r) {
        if ((double)v >= th || r == rm) {
            if (pos < capacity) {
                cand_d[pos] = (int)d;
                cand_r[pos] = (int)r;
            } else {
                rspi_flag(err, RSPI_ERR_CAPACITY);
            }
            ++pos;
        }
    };
    // eight rows' loads in flight per thread, taken in row order
    long long r = ty;
    for (; r + 7 * RY < n_rows; r += 8 * RY) {
        float v8[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v8[u] = __ldg(&ll[(r + u * RY) * stride + x]);
#pragma unroll
        for (int u = 0; u < 8; ++u) take(v8[u], r + u * RY);
    }
    for (; r < n_rows; r += RY) take(ll[r * stride + x], r);
}

// One warp per frame whose threads of k_cand_count each found at most two
// candidates: the recorded rows written in the order k_cand_fill writes them
// (thread ty's rows, ty ascending), so both paths give the same list.
__global__ void k_cand_compact(const int *__restrict__ cand_slot, const int *__restrict__ cnt_part,
                               const long long *__restrict__ cand_off, long long n_data,
                               long long capacity, int *__restrict__ cand_d,
                               int *__restrict__ cand_r, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n_data; d += nwarp) {
        const int slot = cand_slot[d * RY + lane];
        if (__any_sync(RSPI_FULL_MASK, slot == -2)) continue;   // k_cand_fill's frame
        const int v = cnt_part[d * RY + lane];
        const int c = cnt_count(v);
        int pre = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(RSPI_FULL_MASK, pre, o);
            if (lane >= o) pre += u;
        }
        for (int k = 0; k < c; ++k) {
            const long long pos = cand_off[d] + pre - c + k;
            if (pos < capacity) {
                cand_d[pos] = (int)d;
                cand_r[pos] = k == 0 ? slot : lane + RY * (v >> 2);
            } else {
                rspi_flag(err, RSPI_ERR_CAPACITY);
            }
        }
    }
}

// Candidates regrouped by likelihood row: count, scan (rows + 1 offsets),
// scatter of pair indices.  Order within a row does not affect any value.
__global__ void k_row_count(const int *__restrict__ cand_r, const long long *__restrict__ total_ptr,
                            long long capacity, int *__restrict__ row_cnt) {
    const long long total = min(*total_ptr, capacity);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
        atomicAdd(&row_cnt[cand_r[i]], 1);
}

__global__ void k_row_scatter(const int *__restrict__ cand_r, const long long *__restrict__ total_ptr,
                              long long capacity, const long long *__restrict__ row_off,
                              int *__restrict__ cursor, int *__restrict__ row_cand) {
    const long long total = min(*total_ptr, capacity);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int r = cand_r[i];
        row_cand[row_off[r] + atomicAdd(&cursor[r], 1)] = (int)i;
    }
}

// A "direct" row: at most DIRECT_MAX candidates whose entry slots together
// read no more values than the row holds (16 measured faster than 4 at the
// argmax-only window of a 185^2 detector).  Its candidates are evaluated by
// k_rescore_direct, one warp per candidate anywhere on the GPU, each value
// computed with rot_log_value where the sum reads it; k_rescore_rows skips
// the row.  (With about one candidate per row, the argmax-only window's
// usual case, a CTA per row kept one warp of the SM busy.)
constexpr int DIRECT_MAX = 16;

__device__ __forceinline__ bool row_direct(long long r, const long long *__restrict__ row_off,
                                           const int *__restrict__ row_cand,
                                           const int *__restrict__ cand_d,
                                           const long long *__restrict__ row_off32,
                                           long long p_pad) {
    const long long a = row_off[r], b = row_off[r + 1];
    if (a == b || b - a > DIRECT_MAX) return false;
    long long wk = 0;
    for (long long i = a; i < b; ++i) {
        const int d = cand_d[row_cand[i]];
        wk += (row_off32[d + 1] - row_off32[d]) * 32;
    }
    return wk <= p_pad;
}

// One warp per candidate pair of a direct row: the FP64 form's sum (per
// lane over the frame's packed rows, fma(count, L, acc), then the warp
// reduction) with each value from rot_log_value, the same bits as the row
// kernel's.
__global__ void __launch_bounds__(256)
k_rescore_direct(const int *__restrict__ cand_d, const int *__restrict__ cand_r,
                 const long long *__restrict__ total_ptr, long long capacity,
                 const long long *__restrict__ row_off, const int *__restrict__ row_cand,
                 const double *__restrict__ holo, long long num_rot,
                 const double *__restrict__ rot_cs, int size, const double *__restrict__ bg,
                 const int *__restrict__ sel_pix, long long n_sel, long long p_pad,
                 const double *__restrict__ init, const double *__restrict__ scales,
                 const unsigned int *__restrict__ ent32, const long long *__restrict__ row_off32,
                 double *__restrict__ cand_ll, float *__restrict__ ll32, long long ll_stride,
                 const int *__restrict__ col_of_frame) {
    const long long total = min(*total_ptr, capacity);
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long npix = (long long)size * size;
    const float inv_size = 1.f / (float)size;
    for (long long i = warp; i < total; i += nwarp) {
        const long long r = cand_r[i];
        if (!row_direct(r, row_off, row_cand, cand_d, row_off32, p_pad)) continue;   // per warp
        const int d = cand_d[i];
        const long long s0 = r / num_rot, j = r - s0 * num_rot;
        const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
        const double *w = holo + s0 * npix;
        double acc = 0.;
        const unsigned *ep = ent32 + row_off32[d] * 32 + lane;
        for (long long q = row_off32[d]; q < row_off32[d + 1]; ++q, ep += 32) {
            const unsigned e = __ldg(ep);
            const unsigned c = e >> 16;
            double v = 0.;
            if (c < (unsigned)n_sel) {
                const int p = sel_pix[c];
                int x, y;
                pixel_xy(p, size, inv_size, x, y);
                v = rot_log_value(w, x, y, size, ac, as, bg[p]);
            }
            acc = fma((double)(e & 0xffffu), v, acc);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            const double v = init[s0] * scales[d] + acc;
            cand_ll[i] = v;
            ll32[r * ll_stride + (col_of_frame ? col_of_frame[d] : d)] = (float)v;
        }
    }
}

// One CTA per likelihood row with candidates: the row's FP64 rotated slice
// is computed into shared memory with rot_log_value (as k_rot_log_js does),
// then each warp rescores candidate frames exactly as the FP64 form sums
// them (per lane over the frame's packed rows, fma(count, L, acc), then the
// warp reduction), so every value equals the FP64 form's.  A row longer than
// shared memory holds (GROW: more than ~28,100 likelihood pixels) is built
// in the CTA's slot of a global scratch array instead and gathered through
// L1/L2; the arithmetic is the same.  A shared-memory row whose
// candidates' warps read fewer values each than the CTA's threads would
// build (a sparse frame or two, the usual case of the argmax-only window)
// is not built: each value is computed with rot_log_value where the sum
// reads it.
template <bool GROW>
__global__ void __launch_bounds__(1024)
k_rescore_rows(const long long *__restrict__ row_off, const int *__restrict__ row_cand,
               long long n_rows, const int *__restrict__ cand_d, const double *__restrict__ holo,
               long long num_rot, const double *__restrict__ rot_cs, int size,
               const double *__restrict__ bg, const int *__restrict__ sel_pix, long long n_sel,
               long long p_pad, const double *__restrict__ init, const double *__restrict__ scales,
               const unsigned int *__restrict__ ent32, const long long *__restrict__ row_off32,
               double *__restrict__ cand_ll, float *__restrict__ ll32, long long ll_stride,
               const int *__restrict__ col_of_frame, double *row_scratch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sl = GROW ? row_scratch + (long long)blockIdx.x * p_pad
                      : reinterpret_cast<double *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const long long npix = (long long)size * size;
    const unsigned cmax = (unsigned)p_pad - 1;
    const float inv_size = 1.f / (float)size;
    __shared__ long long s_work;
    __shared__ int s_rows[1024], s_cnt[32];
    const long long step = gridDim.x;
    // the CTA's rows r = blockIdx.x + k gridDim.x, taken blockDim.x at a
    // time: each thread tests one (empty rows and k_rescore_direct's rows
    // are skipped) and the rows to build are listed in row order
    for (long long base = blockIdx.x; base < n_rows; base += step * blockDim.x) {
    const long long rt = base + (long long)threadIdx.x * step;
    bool build = false;
    if (rt < n_rows) {
        build = row_off[rt] != row_off[rt + 1];
        if (!GROW && build) build = !row_direct(rt, row_off, row_cand, cand_d, row_off32, p_pad);
    }
    __syncthreads();            // the previous list's readers are done
    const unsigned bal = __ballot_sync(RSPI_FULL_MASK, build);
    if (lane == 0) s_cnt[wid] = __popc(bal);
    __syncthreads();
    int before = 0, n_build = 0;
    for (int k = 0; k < nw; ++k) {
        if (k < wid) before += s_cnt[k];
        n_build += s_cnt[k];
    }
    if (build) s_rows[before + __popc(bal & ((1u << lane) - 1u))] = (int)rt;
    __syncthreads();
    for (int kr = 0; kr < n_build; ++kr) {
        const long long r = s_rows[kr];
        const long long a = row_off[r], b = row_off[r + 1];
        const long long s0 = r / num_rot, j = r - s0 * num_rot;
        const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
        const double *w = holo + s0 * npix;
        __syncthreads();        // the previous row's readers are done
        // the values the row's candidates read (their entry slots): when
        // their warps finish them sooner than the CTA builds the row (work
        // per warp below the row per warp), each is computed where it is
        // read instead (same function, same sums: the same bits).  Rows in
        // global scratch (GROW) are always built: there the candidates of a
        // row are one or two dense frames, and a row left to one warp keeps
        // the SM at one warp in flight (measured slower on a 47,616-pixel
        // row, 10,000 frames).
        bool direct = false;
        if constexpr (!GROW) {
            if (wid == 0) {
                long long wk = 0;
                for (long long i = a + lane; i < b; i += 32) {
                    const int d = cand_d[row_cand[i]];
                    wk += (row_off32[d + 1] - row_off32[d]) * 32;
                }
                wk = warp_sum(wk);
                if (lane == 0) s_work = wk;
            }
            __syncthreads();
            direct = s_work * nw < p_pad * min(b - a, (long long)nw);
        }
        if (!direct) {
            for (long long c = threadIdx.x; c < p_pad; c += blockDim.x) {
                double v = 0.;
                if (c < n_sel) {
                    const int p = sel_pix[c];
                    int x, y;
                    pixel_xy(p, size, inv_size, x, y);
                    v = rot_log_value(w, x, y, size, ac, as, bg[p]);
                }
                sl[c] = v;
            }
        }
        __syncthreads();
        // the likelihood-pixel value of entry column c (0 past n_sel, as
        // the row holds it)
        auto value = [&](unsigned c) -> double {
            if (!direct) return sl[min(c, cmax)];
            if (c >= (unsigned)n_sel) return 0.;
            const int p = sel_pix[c];
            int x, y;
            pixel_xy(p, size, inv_size, x, y);
            return rot_log_value(w, x, y, size, ac, as, bg[p]);
        };
        const double ini = init[s0];
        if constexpr (GROW) {
            // a row in global scratch has a few candidates (dense frames):
            // one warp per candidate
            for (long long i = a + wid; i < b; i += nw) {
                const int pair = row_cand[i];
                const int d = cand_d[pair];
                double acc = 0.;
                const unsigned *ep = ent32 + row_off32[d] * 32 + lane;
                for (long long q = row_off32[d]; q < row_off32[d + 1]; ++q, ep += 32) {
                    const unsigned e = __ldg(ep);
                    acc = fma((double)(e & 0xffffu), value(e >> 16), acc);
                }
                acc = warp_sum(acc);
                if (lane == 0) {
                    const double v = ini * scales[d] + acc;
                    cand_ll[pair] = v;
                    ll32[r * ll_stride + (col_of_frame ? col_of_frame[d] : d)] = (float)v;
                }
            }
        } else {
            // the warp's candidates are a + wid + k nw, k = 0, 1, ...; lane l
            // fetches the metadata of the warp's (k0 + l)-th candidate, so the
            // dependent loads (row_cand -> cand_d -> row_off32) run once per 32
            // candidates instead of once per candidate
            for (long long k0 = 0; a + wid + k0 * nw < b; k0 += 32) {
                const long long il = a + wid + (k0 + lane) * nw;
                int pair = 0, d = 0;
                long long q0 = 0, q1 = 0;
                if (il < b) {
                    pair = row_cand[il];
                    d = cand_d[pair];
                    q0 = row_off32[d];
                    q1 = row_off32[d + 1];
                }
                const int nc = (int)min(32LL, (b - 1 - (a + wid + k0 * nw)) / nw + 1);
                for (int c = 0; c < nc; ++c) {
                    const long long cq0 = __shfl_sync(RSPI_FULL_MASK, q0, c);
                    const long long cq1 = __shfl_sync(RSPI_FULL_MASK, q1, c);
                    double acc = 0.;
                    const unsigned *ep = ent32 + cq0 * 32 + lane;
                    for (long long q = cq0; q < cq1; ++q, ep += 32) {
                        const unsigned e = __ldg(ep);
                        acc = fma((double)(e & 0xffffu), value(e >> 16), acc);
                    }
                    acc = warp_sum(acc);
                    if (lane == c) {
                        const double v = ini * scales[d] + acc;
                        cand_ll[pair] = v;
                        ll32[r * ll_stride + (col_of_frame ? col_of_frame[d] : d)] = (float)v;
                    }
                }
            }
        }
    }
    }
}

// Per frame over its candidates (one warp per frame): first-index argmax,
// max and log-sum-exp.
__global__ void k_cand_finalize(const long long *__restrict__ cand_off,
                                const int *__restrict__ cand_r, const double *__restrict__ cand_ll,
                                const double *__restrict__ max32, const double *__restrict__ noncand,
                                long long n_data, long long capacity, double *__restrict__ maxll,
                                int *__restrict__ rmax, double *__restrict__ logz) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n_data; d += nwarp) {
        const long long a = cand_off[d], b = min(cand_off[d + 1], capacity);
        double m = -INFINITY;
        int idx = 0x7fffffff;
        for (long long i = a + lane; i < b; i += 32) {
            const double v = cand_ll[i];
            if (argmax_better(v, cand_r[i], m, idx)) {
                m = v;
                idx = cand_r[i];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double om = __shfl_xor_sync(RSPI_FULL_MASK, m, o);
            const int oi = __shfl_xor_sync(RSPI_FULL_MASK, idx, o);
            if (argmax_better(om, oi, m, idx)) {
                m = om;
                idx = oi;
            }
        }
        double s = 0.;
        for (long long i = a + lane; i < b; i += 32) s += exp(cand_ll[i] - m);
        s = warp_sum(s);
        if (lane == 0) {
            s += noncand[d] * exp(max32[d] - m);
            maxll[d] = m;
            rmax[d] = b > a ? idx : -1;
            logz[d] = m + log(s);
        }
    }
}

// Scan of per-frame candidate counts (one CTA), with the total at [n].
__global__ void __launch_bounds__(1024)
k_scan_counts(const int *__restrict__ cnt, long long n, long long *__restrict__ off) {
    __shared__ long long part[1024];
    const long long per = (n + 1023) / 1024;
    const long long lo = (long long)threadIdx.x * per, hi = min(n, lo + per);
    long long s = 0;
    for (long long i = lo; i < hi; ++i) s += cnt[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long acc = 0;
        for (int k = 0; k < 1024; ++k) {
            long long v = part[k];
            part[k] = acc;
            acc += v;
        }
        off[n] = acc;
    }
    __syncthreads();
    long long acc = part[threadIdx.x];
    for (long long i = lo; i < hi; ++i) {
        off[i] = acc;
        acc += cnt[i];
    }
}

}  // namespace

extern "C" int rspi_ll16_entry_rows(const int *ones, const int *multi,
                                    const long long *ones_accum, const long long *multi_accum,
                                    const int *place_ones, const int *place_multi,
                                    const int *count_multi, const int *pix2sel, long long num_pix,
                                    long long n_data, int p_zero, int *frame_rows, int *err,
                                    cudaStream_t stream) {
    if (n_data <= 0 || num_pix <= 0 || !frame_rows || !pix2sel || p_zero < 0 ||
        p_zero % 32 || p_zero + 32 > 65536)
        return RSPI_ERR_ARG;
    k_entry16_rows<<<rspi_blocks(n_data * 32, ENTRY_WARPS * 32), ENTRY_WARPS * 32, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, pix2sel,
        num_pix, n_data, p_zero, frame_rows, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_ll16_entry_fill(const int *ones, const int *multi,
                                    const long long *ones_accum, const long long *multi_accum,
                                    const int *place_ones, const int *place_multi,
                                    const int *count_multi, const int *pix2sel, long long num_pix,
                                    long long n_data, int p_zero, const long long *row_off,
                                    unsigned short *entries, cudaStream_t stream) {
    if (n_data <= 0 || num_pix <= 0 || !row_off || !entries || !pix2sel || p_zero < 0 ||
        p_zero % 32 || p_zero + 32 > 65536)
        return RSPI_ERR_ARG;
    k_entry16_fill<<<rspi_blocks(n_data * 32, ENTRY_WARPS * 32), ENTRY_WARPS * 32, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, pix2sel,
        num_pix, n_data, p_zero, row_off, entries);
    RSPI_RETURN_LAUNCH();
}

namespace {

// Candidate selection over a likelihood matrix with n_x columns of stride
// `stride`; column x holds frame frame_of_col[x] (-1: none), or frame x when
// frame_of_col is null.
int candidates_launch(const float *ll, long long n_rows, long long n_x, long long stride,
                      const int *frame_of_col, long long n_data, const double *max32,
                      const int *rmax32, const long long *frame_photons,
                      const long long *row_off16, const float *lmax, double delta,
                      int *cnt_part, int *cand_n, double *noncand, double *thr,
                      long long *cand_off, long long capacity, int *cand_d, int *cand_r,
                      int *err, cudaStream_t stream, int *cand_slot = nullptr) {
    if (!ll || !max32 || !rmax32 || !frame_photons || !row_off16 || !lmax || !cnt_part ||
        !cand_n || !noncand || !thr || !cand_off || !cand_d || !cand_r || n_rows <= 0 ||
        n_data <= 0 || n_x <= 0 || stride < n_x || n_rows > 0x7fffffffLL || capacity < 0 ||
        capacity > 0x7fffffffLL || !(delta >= 0.))
        return RSPI_ERR_ARG;
    const dim3 block(32, RY);
    const unsigned grid = (unsigned)((n_x + 31) / 32);
    k_cand_count<<<grid, block, 0, stream>>>(ll, n_rows, n_x, stride, frame_of_col, max32,
                                             rmax32, frame_photons, row_off16, lmax, delta,
                                             cnt_part, cand_n, noncand, thr, cand_slot);
    k_scan_counts<<<1, 1024, 0, stream>>>(cand_n, n_data, cand_off);
    if (cand_slot)
        k_cand_compact<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
            cand_slot, cnt_part, cand_off, n_data, capacity, cand_d, cand_r, err);
    k_cand_fill<<<grid, block, 0, stream>>>(ll, n_rows, n_x, stride, frame_of_col, cand_slot,
                                            thr, rmax32, cnt_part, cand_off, capacity, cand_d,
                                            cand_r, err);
    RSPI_RETURN_LAUNCH();
}

}  // namespace

extern "C" int rspi_screen_candidates(const float *ll, long long n_rows, long long n_data,
                                      const double *max32, const int *rmax32,
                                      const long long *frame_photons,
                                      const long long *row_off16, const float *lmax, double delta,
                                      int *cnt_part, int *cand_n, double *noncand, double *thr,
                                      long long *cand_off, long long capacity, int *cand_d,
                                      int *cand_r, int *err, cudaStream_t stream) {
    return candidates_launch(ll, n_rows, n_data, n_data, nullptr, n_data, max32, rmax32,
                             frame_photons, row_off16, lmax, delta, cnt_part, cand_n, noncand,
                             thr, cand_off, capacity, cand_d, cand_r, err, stream);
}

extern "C" int rspi_screen_candidates_cols(const float *ll, long long n_rows, long long n_cols,
                                           const int *frame_of_col, long long n_data,
                                           const double *max32, const int *rmax32,
                                           const long long *frame_photons,
                                           const long long *row_off16, const float *lmax,
                                           double delta, int *cnt_part, int *cand_n,
                                           double *noncand, double *thr, long long *cand_off,
                                           long long capacity, int *cand_d, int *cand_r,
                                           int *cand_slot, int *err, cudaStream_t stream) {
    if (!frame_of_col) return RSPI_ERR_ARG;
    return candidates_launch(ll, n_rows, n_cols, n_cols, frame_of_col, n_data, max32, rmax32,
                             frame_photons, row_off16, lmax, delta, cnt_part, cand_n, noncand,
                             thr, cand_off, capacity, cand_d, cand_r, err, stream, cand_slot);
}

static int rescore_launch(const int *cand_d, const int *cand_r, const long long *cand_off,
                            long long n_data, long long capacity, long long n_rows,
                            const double *holo, long long num_rot, const double *rot_cs,
                            long long size, const double *bg, const int *sel_pix, long long n_sel,
                            long long p_pad, const double *init, const double *scales,
                            const unsigned int *entries32, const long long *row_off32,
                            int *row_cnt, long long *row_cand_off, int *row_cand,
                            double *cand_ll, float *ll32, const double *max32,
                            const double *noncand, double *maxll, int *rmax, double *logz,
                            double *row_scratch, long long scratch_rows,
                            const int *col_of_frame, long long ll_stride, cudaStream_t stream) {
    if (!cand_d || !cand_r || !cand_off || !holo || !rot_cs || !bg || !sel_pix || !init ||
        !scales || !entries32 || !row_off32 || !row_cnt || !row_cand_off || !row_cand ||
        !cand_ll || !ll32 || !max32 || !noncand || !maxll || !rmax || !logz || n_data <= 0 ||
        capacity < 0 || capacity > 0x7fffffffLL || n_rows <= 0 || n_rows > 0x7fffffffLL ||
        size <= 1 || size > 46340 || ll_stride < n_data ||
        p_pad < n_sel || p_pad % 32 || p_pad > 65536)
        return RSPI_ERR_ARG;
    const size_t smem = (size_t)p_pad * sizeof(double);
    const bool grow = smem > (size_t)SMEM_LIMIT - 7 * 1024;   // 220 KB: with the static row list
    if (grow && (!row_scratch || scratch_rows < 1)) return RSPI_ERR_ARG;
    static RspiSmemOptIn optin;
    if (!grow && !rspi_smem_optin((const void *)k_rescore_rows<false>, smem, optin))
        return RSPI_ERR_CUDA;
    const long long *total = cand_off + n_data;
    cudaMemsetAsync(row_cnt, 0, sizeof(int) * n_rows, stream);
    k_row_count<<<rspi_sm_count() * 8, 256, 0, stream>>>(cand_r, total, capacity, row_cnt);
    k_scan_counts<<<1, 1024, 0, stream>>>(row_cnt, n_rows, row_cand_off);
    cudaMemsetAsync(row_cnt, 0, sizeof(int) * n_rows, stream);
    k_row_scatter<<<rspi_sm_count() * 8, 256, 0, stream>>>(cand_r, total, capacity, row_cand_off,
                                                          row_cnt, row_cand);
    if (grow) {
        // one CTA per scratch row slot
        const unsigned grid = (unsigned)min(scratch_rows, n_rows);
        k_rescore_rows<true><<<grid, 1024, 0, stream>>>(
            row_cand_off, row_cand, n_rows, cand_d, holo, num_rot, rot_cs, (int)size, bg,
            sel_pix, n_sel, p_pad, init, scales, entries32, row_off32, cand_ll, ll32, ll_stride,
            col_of_frame, row_scratch);
    } else {
        k_rescore_direct<<<rspi_sm_count() * 8, 256, 0, stream>>>(
            cand_d, cand_r, total, capacity, row_cand_off, row_cand, holo, num_rot, rot_cs,
            (int)size, bg, sel_pix, n_sel, p_pad, init, scales, entries32, row_off32, cand_ll,
            ll32, ll_stride, col_of_frame);
        const int per_sm = max(1, (int)(SMEM_LIMIT / (smem + 1024)));
        const unsigned grid = (unsigned)min((long long)rspi_sm_count() * min(per_sm, 2), n_rows);
        k_rescore_rows<false><<<grid, 1024 / min(per_sm, 2), smem, stream>>>(
            row_cand_off, row_cand, n_rows, cand_d, holo, num_rot, rot_cs, (int)size, bg,
            sel_pix, n_sel, p_pad, init, scales, entries32, row_off32, cand_ll, ll32, ll_stride,
            col_of_frame, nullptr);
    }
    k_cand_finalize<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
        cand_off, cand_r, cand_ll, max32, noncand, n_data, capacity, maxll, rmax, logz);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rescore(const int *cand_d, const int *cand_r, const long long *cand_off,
                            long long n_data, long long capacity, long long n_rows,
                            const double *holo, long long num_rot, const double *rot_cs,
                            long long size, const double *bg, const int *sel_pix, long long n_sel,
                            long long p_pad, const double *init, const double *scales,
                            const unsigned int *entries32, const long long *row_off32,
                            int *row_cnt, long long *row_cand_off, int *row_cand,
                            double *cand_ll, float *ll32, const double *max32,
                            const double *noncand, double *maxll, int *rmax, double *logz,
                            double *row_scratch, long long scratch_rows, cudaStream_t stream) {
    return rescore_launch(cand_d, cand_r, cand_off, n_data, capacity, n_rows, holo, num_rot,
                          rot_cs, size, bg, sel_pix, n_sel, p_pad, init, scales, entries32,
                          row_off32, row_cnt, row_cand_off, row_cand, cand_ll, ll32, max32,
                          noncand, maxll, rmax, logz, row_scratch, scratch_rows, nullptr, n_data,
                          stream);
}

extern "C" int rspi_rescore_cols(const int *cand_d, const int *cand_r, const long long *cand_off,
                                 long long n_data, long long capacity, long long n_rows,
                                 const double *holo, long long num_rot, const double *rot_cs,
                                 long long size, const double *bg, const int *sel_pix,
                                 long long n_sel, long long p_pad, const double *init,
                                 const double *scales, const unsigned int *entries32,
                                 const long long *row_off32, int *row_cnt,
                                 long long *row_cand_off, int *row_cand, double *cand_ll,
                                 float *ll32, long long n_cols, const int *col_of_frame,
                                 const double *max32, const double *noncand, double *maxll,
                                 int *rmax, double *logz, double *row_scratch,
                                 long long scratch_rows, cudaStream_t stream) {
    if (!col_of_frame) return RSPI_ERR_ARG;
    return rescore_launch(cand_d, cand_r, cand_off, n_data, capacity, n_rows, holo, num_rot,
                          rot_cs, size, bg, sel_pix, n_sel, p_pad, init, scales, entries32,
                          row_off32, row_cnt, row_cand_off, row_cand, cand_ll, ll32, max32,
                          noncand, maxll, rmax, logz, row_scratch, scratch_rows, col_of_frame,
                          n_cols, stream);
}

// ---------------------------------------------------------------------------
// Candidate selection that allocates nothing
// ---------------------------------------------------------------------------
// rspi_screen_candidates needs n_data * 32 ints of scratch from its caller.
// Some callers cannot provide it: code that runs where it may not call
// cudaMalloc (for example a host thread inside a real-time loop that must
// never block on the driver's allocator, or an application whose device
// memory is all owned by another framework's pool that this library cannot
// draw from).  For them the scratch lives in a fixed file-scope device array
// of NOALLOC_MAX_FRAMES * 32 ints (8 MiB), which every GPU that loads this
// library keeps until the process exits.  The first call on each device
// looks up the array's device address with cudaGetSymbolAddress, with that
// device current; make that first call before any stream capture.  Every
// call on a device shares the one array and it keeps the last call's
// contents: calls whose work overlaps on the GPU (different streams, or two
// host threads) race on it and must be serialised by the caller.  The
// kernels overwrite every scratch entry they later read, so nothing has to
// start at zero.
namespace {

constexpr long long NOALLOC_MAX_FRAMES = 65536;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) int g_cand_scratch[NOALLOC_MAX_FRAMES * RY];

// The array's device address on the current device, looked up once per
// device and cached for the life of the process's primary context (a
// cudaDeviceReset invalidates it; this library is not meant to outlive one).
// Two host threads making the first call on one device at once both look
// the address up and store the same value; the store is atomic.
int *cand_scratch_address(int *status) {
    static std::atomic<int *> addr[NOALLOC_MAX_DEVICES];
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        *status = RSPI_ERR_CUDA;
        return nullptr;
    }
    int *cached = addr[dev].load(std::memory_order_acquire);
    if (cached == nullptr) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_cand_scratch) != cudaSuccess || p == nullptr) {
            *status = RSPI_ERR_CUDA;
            return nullptr;
        }
        cached = static_cast<int *>(p);
        addr[dev].store(cached, std::memory_order_release);
    }
    return cached;
}

}  // namespace

extern "C" int rspi_screen_candidates_noalloc(const float *ll, long long n_rows, long long n_data,
                                              const double *max32, const int *rmax32,
                                              const long long *frame_photons,
                                              const long long *row_off16, const float *lmax,
                                              double delta, int *cand_n, double *noncand,
                                              double *thr, long long *cand_off, long long capacity,
                                              int *cand_d, int *cand_r, int *err,
                                              cudaStream_t stream) {
    if (n_data > NOALLOC_MAX_FRAMES) return RSPI_ERR_TOO_LARGE;
    if (!ll || !max32 || !rmax32 || !frame_photons || !row_off16 || !lmax || !cand_n ||
        !noncand || !thr || !cand_off || !cand_d || !cand_r || n_rows <= 0 || n_data <= 0 ||
        n_rows > 0x7fffffffLL || capacity < 0 || capacity > 0x7fffffffLL || !(delta >= 0.))
        return RSPI_ERR_ARG;
    int status = RSPI_OK;
    int *scratch = cand_scratch_address(&status);
    if (scratch == nullptr) return status;
    const dim3 block(32, RY);
    const unsigned grid = (unsigned)((n_data + 31) / 32);
    k_cand_count<<<grid, block, 0, stream>>>(ll, n_rows, n_data, n_data, nullptr, max32, rmax32,
                                             frame_photons, row_off16, lmax, delta, scratch,
                                             cand_n, noncand, thr, nullptr);
    k_scan_counts<<<1, 1024, 0, stream>>>(cand_n, n_data, cand_off);
    k_cand_fill<<<grid, block, 0, stream>>>(ll, n_rows, n_data, n_data, nullptr, nullptr, thr,
                                            rmax32, scratch, cand_off, capacity, cand_d, cand_r,
                                            err);
    RSPI_RETURN_LAUNCH();
}
