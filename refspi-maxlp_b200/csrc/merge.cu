// Posterior-weighted merge (row a10).
//
// The reference ships, but never launches, merge_all (kernels.cu:139-152: a
// posterior-weighted photon scatter, view[pix] += prob * count) and
// slice_merge (kernels.cu:84-114: the adjoint of the bilinear rotation).
// Composed, they give the standard EMC intensity update per (shift,
// diameter) state s0:
//   num[s0](q) = sum_j R_j^T [ sum_d P[s0,j,d] K_d ](q)
//   den[s0](q) = sum_j w[s0,j] C_j(q),   w[r] = sum_d P[r,d] scale_d,
//   C_j = R_j^T 1 (the coverage of rotation j),  intens = num / den,
// counting only posteriors P >= p_min (P_MIN, emc.py:20).  Posteriors come
// from a (frame, row, log-likelihood) list and the per-frame log-sum-exp.
// FP64 accumulators throughout.
#include "rspi_common.cuh"

namespace {

constexpr int RY = 32;

// pairs (d, r, LL) with exp(LL - logz[d]) >= p_min, from a full FP64 matrix
__global__ void __launch_bounds__(32 * RY)
k_sig_count(const double *__restrict__ ll, long long n_rows, long long n_data,
            const double *__restrict__ logz, double p_min, int *__restrict__ cnt_part,
            int *__restrict__ cnt) {
    __shared__ int sc[RY][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long d = (long long)blockIdx.x * 32 + tx;
    int c = 0;
    if (d < n_data) {
        const double lz = logz[d];
        for (long long r = ty; r < n_rows; r += RY)
            if (exp(ll[r * n_data + d] - lz) >= p_min) ++c;
        cnt_part[d * RY + ty] = c;
    }
    sc[ty][tx] = c;
    __syncthreads();
    if (ty == 0 && d < n_data) {
        int tot = 0;
        for (int k = 0; k < RY; ++k) tot += sc[k][tx];
        cnt[d] = tot;
    }
}

__global__ void __launch_bounds__(32 * RY)
k_sig_fill(const double *__restrict__ ll, long long n_rows, long long n_data,
           const double *__restrict__ logz, double p_min, const int *__restrict__ cnt_part,
           const long long *__restrict__ off, long long capacity, int *__restrict__ pd,
           int *__restrict__ pr, double *__restrict__ pll, int *err) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long d = (long long)blockIdx.x * 32 + tx;
    if (d >= n_data) return;
    long long pos = off[d];
    for (int k = 0; k < ty; ++k) pos += cnt_part[d * RY + k];
    const double lz = logz[d];
    for (long long r = ty; r < n_rows; r += RY) {
        const double v = ll[r * n_data + d];
        if (exp(v - lz) >= p_min) {
            if (pos < capacity) {
                pd[pos] = (int)d;
                pr[pos] = (int)r;
                pll[pos] = v;
            } else {
                rspi_flag(err, RSPI_ERR_CAPACITY);
            }
            ++pos;
        }
    }
}

__global__ void __launch_bounds__(1024)
k_scan_i32(const int *__restrict__ cnt, long long n, long long *__restrict__ off) {
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

// Bilinear footprint of detector pixel (x, y) under rotation (ac, as), the
// geometry of slice_merge (kernels.cu:93-101).  Returns false off-detector.
__device__ __forceinline__ bool footprint(int x, int y, int size, double ac, double as, int &ix,
                                          int &iy, double &fx, double &fy) {
    const int cen = size / 2;
    const double xc = (double)(x - cen), yc = (double)(y - cen);
    const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
    const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
    const double fxl = floor(tx), fyl = floor(ty);
    if (fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2) return false;
    ix = (int)fxl;
    iy = (int)fyl;
    fx = tx - fxl;
    fy = ty - fyl;
    return true;
}

__device__ __forceinline__ void scatter4(double *__restrict__ acc, int size, int ix, int iy,
                                         double fx, double fy, double v) {
    const double cx = 1. - fx, cy = 1. - fy;
    double *a = acc + (long long)ix * size + iy;
    atomicAdd(a, v * cx * cy);
    atomicAdd(a + size, v * fx * cy);
    atomicAdd(a + 1, v * cx * fy);
    atomicAdd(a + size + 1, v * fx * fy);
}

// One warp per significant pair: scatter P * K_d back through rotation j
// into num[s0] and add P * scale_d to w[r].
__global__ void __launch_bounds__(256)
k_merge_scatter(const int *__restrict__ pd, const int *__restrict__ pr,
                const double *__restrict__ pll, const long long *__restrict__ total_ptr,
                long long capacity, const double *__restrict__ logz, double p_min,
                const double *__restrict__ scales, const int *__restrict__ ones,
                const int *__restrict__ multi, const long long *__restrict__ ones_accum,
                const long long *__restrict__ multi_accum, const int *__restrict__ place_ones,
                const int *__restrict__ place_multi, const int *__restrict__ count_multi,
                long long num_rot, const double *__restrict__ rot_cs, int size,
                double *__restrict__ num, double *__restrict__ w) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long total = min(*total_ptr, capacity);
    const long long npix = (long long)size * size;
    for (long long i = warp; i < total; i += nwarp) {
        const int d = pd[i], r = pr[i];
        const double p = exp(pll[i] - logz[d]);
        if (!(p >= p_min)) continue;
        const long long s0 = r / num_rot, j = r - s0 * num_rot;
        const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
        double *acc = num + s0 * npix;
        if (lane == 0) atomicAdd(&w[r], p * scales[d]);
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
        for (int k = lane; k < n_o + n_m; k += 32) {
            int pix;
            double cnt;
            if (k < n_o) {
                pix = place_ones[oa + k];
                cnt = 1.;
            } else {
                pix = place_multi[ma + k - n_o];
                cnt = (double)count_multi[ma + k - n_o];
            }
            if (pix < 0 || pix >= npix) continue;
            int ix, iy;
            double fx, fy;
            if (footprint(pix / size, pix % size, size, ac, as, ix, iy, fx, fy))
                scatter4(acc, size, ix, iy, fx, fy, p * cnt);
        }
    }
}

// Coverage C_j = R_j^T 1 of every rotation (independent of the data).
__global__ void k_coverage(long long num_rot, const double *__restrict__ rot_cs, int size,
                           double *__restrict__ cov) {
    const long long npix = (long long)size * size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < num_rot * npix;
         i += stride) {
        const long long j = i / npix, t = i - j * npix;
        int ix, iy;
        double fx, fy;
        if (footprint((int)(t / size), (int)(t % size), size, rot_cs[2 * j], rot_cs[2 * j + 1],
                      ix, iy, fx, fy))
            scatter4(cov + j * npix, size, ix, iy, fx, fy, 1.);
    }
}

// den[s0][q] = sum_j w[s0*R + j] C_j(q); intens = num / den (0 where den == 0)
__global__ void k_merge_finalize(const double *__restrict__ num, const double *__restrict__ w,
                                 const double *__restrict__ cov, long long n_states0,
                                 long long num_rot, long long npix, double *__restrict__ den,
                                 double *__restrict__ intens) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_states0 * npix;
         i += stride) {
        const long long s0 = i / npix, q = i - s0 * npix;
        double acc = 0.;
        for (long long j = 0; j < num_rot; ++j) {
            const double wj = w[s0 * num_rot + j];
            if (wj != 0.) acc += wj * cov[j * npix + q];
        }
        den[i] = acc;
        intens[i] = acc > 0. ? num[i] / acc : 0.;
    }
}

}  // namespace

extern "C" int rspi_posterior_pairs(const double *ll, long long n_rows, long long n_data,
                                    const double *logz, double p_min, int *cnt_part, int *cnt,
                                    long long *off, long long capacity, int *pair_d, int *pair_r,
                                    double *pair_ll, int *err, cudaStream_t stream) {
    if (!ll || !logz || !cnt_part || !cnt || !off || !pair_d || !pair_r || !pair_ll ||
        n_rows <= 0 || n_data <= 0 || n_rows > 0x7fffffffLL || capacity < 0)
        return RSPI_ERR_ARG;
    const dim3 block(32, RY);
    const unsigned grid = (unsigned)((n_data + 31) / 32);
    k_sig_count<<<grid, block, 0, stream>>>(ll, n_rows, n_data, logz, p_min, cnt_part, cnt);
    k_scan_i32<<<1, 1024, 0, stream>>>(cnt, n_data, off);
    k_sig_fill<<<grid, block, 0, stream>>>(ll, n_rows, n_data, logz, p_min, cnt_part, off,
                                           capacity, pair_d, pair_r, pair_ll, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_merge_coverage(long long num_rot, const double *rot_cs, long long size,
                                   double *cov, cudaStream_t stream) {
    if (num_rot <= 0 || !rot_cs || !cov || size <= 1 || size > 46340) return RSPI_ERR_ARG;
    cudaMemsetAsync(cov, 0, sizeof(double) * num_rot * size * size, stream);
    k_coverage<<<rspi_blocks(num_rot * size * size, 256, 16), 256, 0, stream>>>(
        num_rot, rot_cs, (int)size, cov);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_merge(const int *pair_d, const int *pair_r, const double *pair_ll,
                          const long long *pair_total, long long capacity, const double *logz,
                          double p_min, const double *scales, const int *ones, const int *multi,
                          const long long *ones_accum, const long long *multi_accum,
                          const int *place_ones, const int *place_multi, const int *count_multi,
                          long long n_states0, long long num_rot, const double *rot_cs,
                          long long size, const double *cov, double *num, double *den,
                          double *w, double *intens, cudaStream_t stream) {
    if (!pair_d || !pair_r || !pair_ll || !pair_total || !logz || !scales || !ones || !multi ||
        !ones_accum || !multi_accum || !rot_cs || !cov || !num || !den || !w || !intens ||
        n_states0 <= 0 || num_rot <= 0 || size <= 1 || size > 46340 || capacity < 0)
        return RSPI_ERR_ARG;
    const long long npix = size * size;
    cudaMemsetAsync(num, 0, sizeof(double) * n_states0 * npix, stream);
    cudaMemsetAsync(w, 0, sizeof(double) * n_states0 * num_rot, stream);
    k_merge_scatter<<<rspi_sm_count() * 8, 256, 0, stream>>>(
        pair_d, pair_r, pair_ll, pair_total, capacity, logz, p_min, scales, ones, multi,
        ones_accum, multi_accum, place_ones, place_multi, count_multi, num_rot, rot_cs,
        (int)size, num, w);
    k_merge_finalize<<<rspi_blocks(n_states0 * npix, 256, 16), 256, 0, stream>>>(
        num, w, cov, n_states0, num_rot, npix, den, intens);
    RSPI_RETURN_LAUNCH();
}
