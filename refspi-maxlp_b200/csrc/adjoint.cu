// Negative log-likelihood of the MaxLP model and its hand-written adjoint
// (row a16).
//
//   NLL = sum_d sum_t [ s_d |F_t + r_dt|^2 - k_dt log(s_d |F_t + r_dt|^2) ]
//   r_dt = ff(pi q_t dia_d) exp(2 pi i (qx_t sx_d + qy_t sy_d))   (maxLP.py:238-243)
//   ff(x) = (sin x - x cos x) / x^3,  ff'(x) = sin x / x^2 - 3 ff(x) / x
//
// over the phaser pixels t (maxLP.py:88) and frames d, with k_dt the photons
// of frame d at t's rotated detector pixel (maxLP.py:245-253; the exact
// forward map of rspi_common.cuh) and per-frame scale s_d.  The reference's
// own gradient (get_grad_pixel, maxLP.py:199-214) is broken; this is the
// build's definition.  Nothing frames x pixels is stored: both kernels
// recompute r_dt wherever they need it.
//
// Dense part (every frame x pixel, no photons): s_d a, a = |z|^2, z = F + r;
//   dF += 2 s_d z, ds_d += a, dp_d += <2 s_d z, dr/dp> for p in dia, sx, sy.
// Photon part (one term per photon and model pixel mapping onto it):
//   -k log(s_d a);  dF -= 2 k z / a, ds_d -= k / s_d, dp_d -= <2 k z / a, dr/dp>.
// CT is the arithmetic type of the terms (float: the production FP32 form;
// double: the FP64 form used by the finite-difference checks); every sum is
// accumulated in FP64.
#include "rspi_common.cuh"

namespace {

constexpr double PI = 3.14159265358979311599796346854;  // the double nearest pi
constexpr int DT_FRAMES = 32;                             // frames per dense tile

template <typename CT>
struct Ref {
    CT rr, ri;            // r
    CT dd_r, dd_i;        // dr/ddia
    CT dx_r, dx_i;        // dr/dsx
    CT dy_r, dy_i;        // dr/dsy
};

__device__ __forceinline__ void sc(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void sc(double x, double *s, double *c) { sincos(x, s, c); }

template <typename CT>
__device__ __forceinline__ Ref<CT> ref_amp(CT qx, CT qy, CT qrad, CT dia, CT sx, CT sy) {
    Ref<CT> o;
    const CT pq = (CT)PI * qrad;
    const CT x = pq * dia;
    CT sn, cs;
    sc(x, &sn, &cs);
    const CT ix = (CT)1 / x;
    const CT ff = (sn - x * cs) * ix * ix * ix;
    const CT dff = sn * ix * ix - (CT)3 * ff * ix;
    const CT th = (CT)(2. * PI) * (qx * sx + qy * sy);
    CT st, ct;
    sc(th, &st, &ct);
    o.rr = ff * ct;
    o.ri = ff * st;
    o.dd_r = dff * pq * ct;
    o.dd_i = dff * pq * st;
    const CT tx = (CT)(2. * PI) * qx, ty = (CT)(2. * PI) * qy;
    o.dx_r = -tx * o.ri;
    o.dx_i = tx * o.rr;
    o.dy_r = -ty * o.ri;
    o.dy_i = ty * o.rr;
    return o;
}

// Dense tile: a CTA of 256 threads covers 256 pixels x DT_FRAMES frames.
template <typename CT, bool GRAD>
__global__ void __launch_bounds__(256)
k_nll_dense(const double *__restrict__ fre, const double *__restrict__ fim,
            const double *__restrict__ qx, const double *__restrict__ qy,
            const double *__restrict__ qrad, long long n_pix, const double *__restrict__ dia,
            const double *__restrict__ sx, const double *__restrict__ sy,
            const double *__restrict__ scale, long long n_frames, double *__restrict__ out,
            double *__restrict__ gfre, double *__restrict__ gfim, double *__restrict__ gdia,
            double *__restrict__ gsx, double *__restrict__ gsy, double *__restrict__ gscale) {
    __shared__ double fsum[DT_FRAMES][4];
    __shared__ double red[32];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long d0 = (long long)blockIdx.y * DT_FRAMES;
    const int lane = threadIdx.x & 31;
    const bool live = t < n_pix;
    if (GRAD)
        for (int i = threadIdx.x; i < DT_FRAMES * 4; i += blockDim.x) fsum[i / 4][i % 4] = 0.;
    __syncthreads();
    const CT f_r = live ? (CT)fre[t] : (CT)0, f_i = live ? (CT)fim[t] : (CT)0;
    const CT q_x = live ? (CT)qx[t] : (CT)0, q_y = live ? (CT)qy[t] : (CT)0;
    const CT q_r = live ? (CT)qrad[t] : (CT)1;
    double nll = 0., gr = 0., gi = 0.;
    for (int k = 0; k < DT_FRAMES; ++k) {
        const long long d = d0 + k;
        if (d >= n_frames) break;
        const CT s = (CT)scale[d];
        double ga = 0., gd = 0., gx = 0., gy = 0.;
        if (live) {
            const Ref<CT> r = ref_amp<CT>(q_x, q_y, q_r, (CT)dia[d], (CT)sx[d], (CT)sy[d]);
            const CT zr = f_r + r.rr, zi = f_i + r.ri;
            const CT a = zr * zr + zi * zi;
            nll += (double)(s * a);
            if (GRAD) {
                const CT wr = (CT)2 * s * zr, wi = (CT)2 * s * zi;   // d(s a)/dz
                gr += (double)wr;
                gi += (double)wi;
                ga = (double)a;
                gd = (double)(wr * r.dd_r + wi * r.dd_i);
                gx = (double)(wr * r.dx_r + wi * r.dx_i);
                gy = (double)(wr * r.dy_r + wi * r.dy_i);
            }
        }
        if (GRAD) {
            ga = warp_sum(ga);
            gd = warp_sum(gd);
            gx = warp_sum(gx);
            gy = warp_sum(gy);
            if (lane == 0) {
                atomicAdd(&fsum[k][0], ga);
                atomicAdd(&fsum[k][1], gd);
                atomicAdd(&fsum[k][2], gx);
                atomicAdd(&fsum[k][3], gy);
            }
        }
    }
    const double tot = block_sum(nll, red);
    if (threadIdx.x == 0) atomicAdd(out, tot);
    if (GRAD) {
        if (live) {
            atomicAdd(&gfre[t], gr);
            atomicAdd(&gfim[t], gi);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < DT_FRAMES; i += blockDim.x) {
            const long long d = d0 + i;
            if (d < n_frames) {
                atomicAdd(&gscale[d], fsum[i][0]);
                atomicAdd(&gdia[d], fsum[i][1]);
                atomicAdd(&gsx[d], fsum[i][2]);
                atomicAdd(&gsy[d], fsum[i][3]);
            }
        }
    }
}

// Photon part: one warp per frame, lanes over its photons; each photon goes
// to every phaser pixel whose exact rotated index lands on it.
template <typename CT, bool GRAD>
__global__ void __launch_bounds__(256)
k_nll_photons(const int *__restrict__ ones, const int *__restrict__ multi,
              const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
              const int *__restrict__ place_ones, const int *__restrict__ place_multi,
              const int *__restrict__ count_multi, long long n_frames,
              const double *__restrict__ rot_cs, int size, const int *__restrict__ mask_idx,
              const double *__restrict__ fre, const double *__restrict__ fim,
              const double *__restrict__ qx, const double *__restrict__ qy,
              const double *__restrict__ qrad, const double *__restrict__ dia,
              const double *__restrict__ sx, const double *__restrict__ sy,
              const double *__restrict__ scale, double *__restrict__ out,
              double *__restrict__ gfre, double *__restrict__ gfim, double *__restrict__ gdia,
              double *__restrict__ gsx, double *__restrict__ gsy, double *__restrict__ gscale,
              int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long npix = (long long)size * size;
    const double c0 = (double)(size / 2);
    double nll = 0.;
    for (long long d = warp; d < n_frames; d += nwarp) {
        const double c = rot_cs[2 * d], s = rot_cs[2 * d + 1];
        const CT sd = (CT)scale[d], dd = (CT)dia[d], xd = (CT)sx[d], yd = (CT)sy[d];
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
        double ga = 0., gd = 0., gx = 0., gy = 0.;
        for (int i = lane; i < n_o + n_m; i += 32) {
            int p, cnt;
            if (i < n_o) {
                p = place_ones[oa + i];
                cnt = 1;
            } else {
                p = place_multi[ma + i - n_o];
                cnt = count_multi[ma + i - n_o];
            }
            if (p < 0 || p >= npix) {
                rspi_flag(err, RSPI_ERR_INDEX);
                continue;
            }
            const int ux = p / size, uy = p - (p / size) * size;
            // model pixels near the inverse image (3x3), checked with the forward map
            const double vx = (double)ux - c0, vy = (double)uy - c0;
            const int bx = (int)rint(c * vx + s * vy + c0);
            const int by = (int)rint(-s * vx + c * vy + c0);
            for (int ax = -1; ax <= 1; ++ax)
                for (int ay = -1; ay <= 1; ++ay) {
                    const int tx = bx + ax, ty = by + ay;
                    if (tx < 0 || ty < 0 || tx >= size || ty >= size) continue;
                    const int m = mask_idx[tx * size + ty];
                    if (m < 0) continue;
                    int ox, oy;
                    forward_pixel(tx, ty, c, s, size, ox, oy);
                    if (ox != ux || oy != uy) continue;
                    const Ref<CT> r = ref_amp<CT>((CT)qx[m], (CT)qy[m], (CT)qrad[m], dd, xd, yd);
                    const CT zr = (CT)fre[m] + r.rr, zi = (CT)fim[m] + r.ri;
                    const CT a = zr * zr + zi * zi;
                    const CT k = (CT)cnt;
                    nll -= (double)k * log((double)(sd * a));
                    if (GRAD) {
                        const CT wr = (CT)2 * k * zr / a, wi = (CT)2 * k * zi / a;
                        atomicAdd(&gfre[m], -(double)wr);
                        atomicAdd(&gfim[m], -(double)wi);
                        ga -= (double)(k / sd);
                        gd -= (double)(wr * r.dd_r + wi * r.dd_i);
                        gx -= (double)(wr * r.dx_r + wi * r.dx_i);
                        gy -= (double)(wr * r.dy_r + wi * r.dy_i);
                    }
                }
        }
        if (GRAD) {
            ga = warp_sum(ga);
            gd = warp_sum(gd);
            gx = warp_sum(gx);
            gy = warp_sum(gy);
            if (lane == 0) {
                atomicAdd(&gscale[d], ga);
                atomicAdd(&gdia[d], gd);
                atomicAdd(&gsx[d], gx);
                atomicAdd(&gsy[d], gy);
            }
        }
    }
    nll = warp_sum(nll);
    if (lane == 0) atomicAdd(out, nll);
}

template <typename CT, bool GRAD>
void launch_all(const int *ones, const int *multi, const long long *oacc, const long long *macc,
                const int *po, const int *pm, const int *cm, long long n_frames,
                const double *rot_cs, int size, const int *mask_idx, long long n_pix,
                const double *fre, const double *fim, const double *qx, const double *qy,
                const double *qrad, const double *dia, const double *sx, const double *sy,
                const double *scale, double *out, double *gfre, double *gfim, double *gdia,
                double *gsx, double *gsy, double *gscale, int *err, cudaStream_t stream) {
    const dim3 grid((unsigned)((n_pix + 255) / 256), (unsigned)((n_frames + DT_FRAMES - 1) / DT_FRAMES));
    if (n_pix > 0)
        k_nll_dense<CT, GRAD><<<grid, 256, 0, stream>>>(fre, fim, qx, qy, qrad, n_pix, dia, sx,
                                                         sy, scale, n_frames, out, gfre, gfim,
                                                         gdia, gsx, gsy, gscale);
    k_nll_photons<CT, GRAD><<<rspi_blocks(n_frames * 32, 256), 256, 0, stream>>>(
        ones, multi, oacc, macc, po, pm, cm, n_frames, rot_cs, size, mask_idx, fre, fim, qx, qy,
        qrad, dia, sx, sy, scale, out, gfre, gfim, gdia, gsx, gsy, gscale, err);
}

}  // namespace

extern "C" int rspi_nll(int precision, int want_grad, const int *ones, const int *multi,
                        const long long *ones_accum, const long long *multi_accum,
                        const int *place_ones, const int *place_multi, const int *count_multi,
                        long long n_frames, const double *rot_cs, long long size,
                        const int *mask_idx, long long n_pix, const double *fre,
                        const double *fim, const double *qx, const double *qy,
                        const double *qrad, const double *dia, const double *sx,
                        const double *sy, const double *scale, double *nll, double *gfre,
                        double *gfim, double *gdia, double *gsx, double *gsy, double *gscale,
                        int *err, cudaStream_t stream) {
    if (n_frames <= 0 || n_frames > 0x7fffffffLL * DT_FRAMES || size <= 1 || size > 46340 ||
        n_pix < 0 || !ones || !multi || !ones_accum || !multi_accum || !rot_cs || !mask_idx ||
        !fre || !fim || !qx || !qy || !qrad || !dia || !sx || !sy || !scale || !nll ||
        (precision != 0 && precision != 1))
        return RSPI_ERR_ARG;
    if (want_grad && (!gfre || !gfim || !gdia || !gsx || !gsy || !gscale)) return RSPI_ERR_ARG;
    cudaMemsetAsync(nll, 0, sizeof(double), stream);
    if (want_grad) {
        cudaMemsetAsync(gfre, 0, sizeof(double) * n_pix, stream);
        cudaMemsetAsync(gfim, 0, sizeof(double) * n_pix, stream);
        cudaMemsetAsync(gdia, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gsx, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gsy, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gscale, 0, sizeof(double) * n_frames, stream);
    }
#define RSPI_NLL(CT, G)                                                                          \
    launch_all<CT, G>(ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, \
                      n_frames, rot_cs, (int)size, mask_idx, n_pix, fre, fim, qx, qy, qrad, dia,  \
                      sx, sy, scale, nll, gfre, gfim, gdia, gsx, gsy, gscale, err, stream)
    if (precision == 1 && want_grad) RSPI_NLL(double, true);
    else if (precision == 1) RSPI_NLL(double, false);
    else if (want_grad) RSPI_NLL(float, true);
    else RSPI_NLL(float, false);
#undef RSPI_NLL
    RSPI_RETURN_LAUNCH();
}
