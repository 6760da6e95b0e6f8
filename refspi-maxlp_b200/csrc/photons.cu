// Photon-list setup (rows a1, a2): prefix sums, per-frame counts, scales,
// powder and the packed likelihood entry lists.  All results are integer or
// exactly representable, so they are bit-exact with dset.py's arithmetic.
#include "rspi_common.cuh"

namespace {

constexpr int SCAN_THREADS = 1024;

// Exclusive prefix sum of int32 counts into int64 (dset.py:32-33,41-42:
// roll(cumsum)) and the total.  One CTA; each thread owns a contiguous run.
__global__ void __launch_bounds__(SCAN_THREADS)
k_exclusive_scan(const int *__restrict__ in, long long n, long long *__restrict__ out,
                 long long *__restrict__ total, int *err) {
    __shared__ long long part[SCAN_THREADS];
    const long long per = (n + SCAN_THREADS - 1) / SCAN_THREADS;
    const long long lo = (long long)threadIdx.x * per;
    const long long hi = min(n, lo + per);
    long long s = 0;
    for (long long i = lo; i < hi; ++i) {
        int v = in[i];
        if (v < 0) rspi_flag(err, RSPI_ERR_INDEX);
        s += v;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long acc = 0;
        for (int k = 0; k < SCAN_THREADS; ++k) {
            long long v = part[k];
            part[k] = acc;
            acc += v;
        }
        if (total) *total = acc;
    }
    __syncthreads();
    long long acc = part[threadIdx.x];
    for (long long i = lo; i < hi; ++i) {
        out[i] = acc;
        acc += in[i];
    }
}

// counts[d] = ones[d] + sum of the frame's multi counts (dset.py:50-53) and
// the grand total of count_multi.  One warp per frame.
__global__ void k_frame_counts(const int *__restrict__ ones, const int *__restrict__ multi,
                               const long long *__restrict__ multi_accum,
                               const int *__restrict__ count_multi, long long n,
                               long long *__restrict__ counts,
                               unsigned long long *__restrict__ total_multi_counts, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n; d += nwarp) {
        const long long a = multi_accum[d];
        const int m = multi[d];
        long long s = 0;
        for (int i = lane; i < m; i += 32) {
            int c = count_multi[a + i];
            if (c < 0) rspi_flag(err, RSPI_ERR_INDEX);
            s += c;
        }
        s = warp_sum(s);
        if (lane == 0) {
            counts[d] = (long long)ones[d] + s;
            atomicAdd(total_multi_counts, (unsigned long long)s);
        }
    }
}

// mean_count (dset.py:46-48) and scales (emc.py:129-132).
__global__ void k_scales(const long long *__restrict__ counts, long long n,
                         const long long *__restrict__ totals, double *__restrict__ mean_count,
                         double *__restrict__ scales, int need_scaling) {
    const double mc = (double)(totals[0] + totals[2]) / (double)n;
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 == 0) *mean_count = mc;
    for (long long d = i0; d < n; d += (long long)gridDim.x * blockDim.x)
        scales[d] = need_scaling ? (double)counts[d] / mc : 1.0;
}

// Sum of photons per pixel; integer sums in FP64 are exact, so the atomics'
// order does not matter (dset.py:74-83, np.add.at).
__global__ void k_powder_add(const int *__restrict__ place_ones, long long n_ones,
                             const int *__restrict__ place_multi,
                             const int *__restrict__ count_multi, long long n_multi,
                             long long num_pix, double *__restrict__ powder, int *err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_ones + n_multi;
         i += stride) {
        int p;
        double c;
        if (i < n_ones) {
            p = place_ones[i];
            c = 1.;
        } else {
            p = place_multi[i - n_ones];
            c = (double)count_multi[i - n_ones];
        }
        if (p < 0 || p >= num_pix) {
            rspi_flag(err, RSPI_ERR_INDEX);
            continue;
        }
        atomicAdd(&powder[p], c);
    }
}

__global__ void k_powder_div(double *__restrict__ powder, long long num_pix, long long n_data) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < num_pix; p += stride)
        powder[p] = powder[p] / (double)n_data;
}

// Entry i of frame d in the ones-then-multi order: sel index (or -1) and count.
struct Entry {
    int c;
    int cnt;
};

__device__ __forceinline__ Entry frame_entry(int i, int n_o, long long oa, long long ma,
                                             const int *place_ones, const int *place_multi,
                                             const int *count_multi, const int *pix2sel,
                                             long long num_pix, int *err) {
    Entry e{-1, 0};
    int p;
    if (i < n_o) {
        p = place_ones[oa + i];
        e.cnt = 1;
    } else {
        p = place_multi[ma + (i - n_o)];
        e.cnt = count_multi[ma + (i - n_o)];
    }
    if (p < 0 || p >= num_pix) {
        rspi_flag(err, RSPI_ERR_INDEX);
        return e;
    }
    e.c = pix2sel[p];
    if (e.c >= 0 && (e.c > 0xffff || e.cnt < 0 || e.cnt > 0xffff)) {
        rspi_flag(err, RSPI_ERR_CAPACITY);
        e.c = -1;
    }
    return e;
}

constexpr int ENTRY_WARPS = 8;

// Pass 1: rows per frame = the largest bank population (bank = sel % 32).
__global__ void __launch_bounds__(ENTRY_WARPS * 32)
k_entry_rows(const int *__restrict__ ones, const int *__restrict__ multi,
             const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
             const int *__restrict__ place_ones, const int *__restrict__ place_multi,
             const int *__restrict__ count_multi, const int *__restrict__ pix2sel,
             long long num_pix, long long n, int *__restrict__ frame_rows,
             long long *__restrict__ frame_sel_photons, int *err) {
    __shared__ int hist[ENTRY_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long nwarp = (long long)gridDim.x * ENTRY_WARPS;
    for (long long d = (long long)blockIdx.x * ENTRY_WARPS + w; d < n; d += nwarp) {
        hist[w][lane] = 0;
        __syncwarp();
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
        long long phot = 0;
        for (int i = lane; i < n_o + n_m; i += 32) {
            Entry e = frame_entry(i, n_o, oa, ma, place_ones, place_multi, count_multi,
                                  pix2sel, num_pix, err);
            if (e.c >= 0) {
                atomicAdd(&hist[w][e.c & 31], 1);
                phot += e.cnt;
            }
        }
        __syncwarp();
        int rows = warp_max_int(hist[w][lane]);
        phot = warp_sum(phot);
        if (lane == 0) {
            frame_rows[d] = rows;
            if (frame_sel_photons) frame_sel_photons[d] = phot;
        }
        __syncwarp();
    }
}

// Pass 2: deterministic placement.  Within each chunk of 32 entries a lane's
// slot in its bank is its rank among same-bank lanes (match_any), so the
// layout depends only on the input order.
__global__ void __launch_bounds__(ENTRY_WARPS * 32)
k_entry_fill(const int *__restrict__ ones, const int *__restrict__ multi,
             const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
             const int *__restrict__ place_ones, const int *__restrict__ place_multi,
             const int *__restrict__ count_multi, const int *__restrict__ pix2sel,
             long long num_pix, long long n, const long long *__restrict__ row_off,
             unsigned int *__restrict__ entries, int *err) {
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
            Entry e{-1, 0};
            if (i < n_o + n_m)
                e = frame_entry(i, n_o, oa, ma, place_ones, place_multi, count_multi, pix2sel,
                                num_pix, nullptr);
            const int key = e.c >= 0 ? (e.c & 31) : 32 + lane;
            const unsigned peers = __match_any_sync(RSPI_FULL_MASK, key);
            const int rank = __popc(peers & lt_mask);
            if (e.c >= 0) {
                const int b = e.c & 31;
                const long long slot = base[w][b] + rank;
                if (slot < nrows)
                    entries[(r0 + slot) * 32 + b] = ((unsigned)e.c << 16) | (unsigned)e.cnt;
                else
                    rspi_flag(err, RSPI_ERR_CAPACITY);
            }
            __syncwarp();
            if (e.c >= 0 && rank == 0) base[w][e.c & 31] += __popc(peers);
            __syncwarp();
        }
        // pad the bank's column with (b << 16 | 0): a zero-count read of a
        // valid slot in the same bank
        for (long long r = base[w][lane]; r < nrows; ++r)
            entries[(r0 + r) * 32 + lane] = ((unsigned)lane << 16);
        __syncwarp();
    }
}

}  // namespace

extern "C" int rspi_photon_offsets(const int *ones, const int *multi, const int *count_multi,
                                   long long n_data, long long *ones_accum,
                                   long long *multi_accum, long long *counts, long long *totals,
                                   double *mean_count, double *scales, int need_scaling,
                                   int *err, cudaStream_t stream) {
    if (n_data <= 0 || !ones || !multi || !ones_accum || !multi_accum || !counts || !totals ||
        !mean_count || !scales || (!count_multi))
        return RSPI_ERR_ARG;
    k_exclusive_scan<<<1, SCAN_THREADS, 0, stream>>>(ones, n_data, ones_accum, totals + 0, err);
    k_exclusive_scan<<<1, SCAN_THREADS, 0, stream>>>(multi, n_data, multi_accum, totals + 1, err);
    cudaMemsetAsync(totals + 2, 0, sizeof(long long), stream);
    k_frame_counts<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
        ones, multi, multi_accum, count_multi, n_data, counts,
        (unsigned long long *)(totals + 2), err);
    k_scales<<<rspi_blocks(n_data, 256), 256, 0, stream>>>(counts, n_data, totals, mean_count,
                                                          scales, need_scaling);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_powder(const int *place_ones, long long n_ones, const int *place_multi,
                           const int *count_multi, long long n_multi, long long num_pix,
                           long long n_data, double *powder, int *err, cudaStream_t stream) {
    if (num_pix <= 0 || n_data <= 0 || !powder || n_ones < 0 || n_multi < 0) return RSPI_ERR_ARG;
    cudaMemsetAsync(powder, 0, sizeof(double) * num_pix, stream);
    if (n_ones + n_multi > 0)
        k_powder_add<<<rspi_blocks(n_ones + n_multi, 256), 256, 0, stream>>>(
            place_ones, n_ones, place_multi, count_multi, n_multi, num_pix, powder, err);
    k_powder_div<<<rspi_blocks(num_pix, 256), 256, 0, stream>>>(powder, num_pix, n_data);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_ll_entry_rows(const int *ones, const int *multi, const long long *ones_accum,
                                  const long long *multi_accum, const int *place_ones,
                                  const int *place_multi, const int *count_multi,
                                  const int *pix2sel, long long num_pix, long long n_data,
                                  int *frame_rows, long long *frame_sel_photons, int *err,
                                  cudaStream_t stream) {
    if (n_data <= 0 || num_pix <= 0 || !frame_rows || !pix2sel) return RSPI_ERR_ARG;
    k_entry_rows<<<rspi_blocks(n_data * 32, ENTRY_WARPS * 32), ENTRY_WARPS * 32, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, pix2sel,
        num_pix, n_data, frame_rows, frame_sel_photons, err);
    RSPI_RETURN_LAUNCH();
}

namespace {
// Exclusive scan of int32 row counts into int64 offsets with the total at [n].
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_rows(const int *__restrict__ rows, long long n, long long *__restrict__ off) {
    __shared__ long long part[SCAN_THREADS];
    const long long per = (n + SCAN_THREADS - 1) / SCAN_THREADS;
    const long long lo = (long long)threadIdx.x * per;
    const long long hi = min(n, lo + per);
    long long s = 0;
    for (long long i = lo; i < hi; ++i) s += rows[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long acc = 0;
        for (int k = 0; k < SCAN_THREADS; ++k) {
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
        acc += rows[i];
    }
}
}  // namespace

extern "C" int rspi_scan_rows(const int *frame_rows, long long n_data, long long *row_off,
                              cudaStream_t stream) {
    if (n_data <= 0 || !frame_rows || !row_off) return RSPI_ERR_ARG;
    k_scan_rows<<<1, SCAN_THREADS, 0, stream>>>(frame_rows, n_data, row_off);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_ll_entry_fill(const int *ones, const int *multi, const long long *ones_accum,
                                  const long long *multi_accum, const int *place_ones,
                                  const int *place_multi, const int *count_multi,
                                  const int *pix2sel, long long num_pix, long long n_data,
                                  const long long *row_off, unsigned int *entries, int *err,
                                  cudaStream_t stream) {
    if (n_data <= 0 || num_pix <= 0 || !row_off || !entries || !pix2sel) return RSPI_ERR_ARG;
    k_entry_fill<<<rspi_blocks(n_data * 32, ENTRY_WARPS * 32), ENTRY_WARPS * 32, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, pix2sel,
        num_pix, n_data, row_off, entries, err);
    RSPI_RETURN_LAUNCH();
}
