// Negative log-likelihood of the EMC likelihood through model slicing, and
// its hand-written adjoint (row a16, the E-step side).
//
// For frame d in its chosen orientation (rotation (cos, sin) of angle
// theta_d) with continuous sphere diameter dia_d, shift (sx_d, sy_d) and
// scale s_d:
//
//   W_d(q)  = |M(q) + r_d(q)|^2 + bg(q)                      (kernels.cu:58-75)
//   r_d(q)  = ff(pi rho_q dia_d / size) exp(2 pi i ((x-c) sx_d + (y-c) sy_d) / size)
//   L_d(p)  = log(bilinear(W_d)(R(theta_d)(p - c) + c) + bg(p))   (kernels.cu:19-41;
//             -1000 outside the detector or below 1e-20, no gradient there)
//   NLL     = sum_d [ vscale s_d sum_{q in sel} W_d(q)
//                     - sum_{p in sel} K_d(p) (log s_d + L_d(p)) ]
//
// i.e. minus the reference's likelihood calc_prob_all (emc.py:194-199,
// kernels.cu:116-137) of each frame in its state, with the Poisson term
// K log s_d that the reference drops (it is the same for every state) kept
// so that the scale has a finite optimum; vscale is a fixed constant.  At
// grid values of (dia, sx, sy, theta), NLL_d = -(LL[state, d] + K_d log s_d).
//
// The adjoint scatters each photon's -K / (B + bg) through the bilinear
// weights to the four model pixels it was interpolated from (the transpose
// of the slicing), and the masked-sum term vscale s_d to every likelihood
// pixel; dW/dM = 2 (M + r), dW/dp = 2 Re(conj(M + r) dr/dp).  Slices are
// recomputed where needed: nothing frames x pixels is stored.  CT is the
// arithmetic type of the terms (float: production; double: the form the
// finite-difference checks use); every sum is FP64.
#include "rspi_common.cuh"

namespace {

constexpr double PI = 3.14159265358979311599796346854;  // the double nearest pi
constexpr int EN_FRAMES = 32;                             // frames per dense tile

__device__ __forceinline__ void scs(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void scs(double x, double *s, double *c) { sincos(x, s, c); }

// r at pixel (x, y) for one frame and its derivatives by dia, sx, sy.
template <typename CT>
struct Holo {
    CT rr, ri, dd_r, dd_i, dx_r, dx_i, dy_r, dy_i;
};

template <typename CT>
__device__ __forceinline__ Holo<CT> holo_ref(int x, int y, int size, CT dia, CT sx, CT sy) {
    const int cen = size / 2;
    const CT dx = (CT)(x - cen), dy = (CT)(y - cen);
    const CT rho = sqrt(dx * dx + dy * dy);
    const CT k = (CT)PI * rho / (CT)size;          // ds / ddia
    CT s = k * dia;
    const bool zero = s == (CT)0;
    if (zero) s = (CT)1.e-5;                       // kernels.cu:66-67
    CT sn, cs;
    scs(s, &sn, &cs);
    const CT is = (CT)1 / s;
    const CT ff = (sn - s * cs) * is * is * is;
    const CT dff = zero ? (CT)0 : sn * is * is - (CT)3 * ff * is;
    const CT th = (CT)(2. * PI) * (dx * sx + dy * sy) / (CT)size;
    CT st, ct;
    scs(th, &st, &ct);
    Holo<CT> h;
    h.rr = ff * ct;
    h.ri = ff * st;
    h.dd_r = dff * k * ct;
    h.dd_i = dff * k * st;
    const CT tx = (CT)(2. * PI) * dx / (CT)size, ty = (CT)(2. * PI) * dy / (CT)size;
    h.dx_r = -tx * h.ri;
    h.dx_i = tx * h.rr;
    h.dy_r = -ty * h.ri;
    h.dy_i = ty * h.rr;
    return h;
}

// Masked-sum term: a CTA covers 256 likelihood pixels x EN_FRAMES frames.
template <typename CT, bool GRAD>
__global__ void __launch_bounds__(256)
k_emc_nll_msum(const double2 *__restrict__ model, int size, const double *__restrict__ bg,
               const int *__restrict__ sel_pix, long long n_sel, const double *__restrict__ dia,
               const double *__restrict__ sx, const double *__restrict__ sy,
               const double *__restrict__ scale, long long n_frames, double vscale,
               double *__restrict__ out, double *__restrict__ gre, double *__restrict__ gim,
               double *__restrict__ gdia, double *__restrict__ gsx, double *__restrict__ gsy,
               double *__restrict__ gscale) {
    __shared__ double fsum[EN_FRAMES][4];
    __shared__ double red[32];
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long d0 = (long long)blockIdx.y * EN_FRAMES;
    const int lane = threadIdx.x & 31;
    const bool live = c < n_sel;
    if (GRAD)
        for (int i = threadIdx.x; i < EN_FRAMES * 4; i += blockDim.x) fsum[i / 4][i % 4] = 0.;
    __syncthreads();
    int p = 0, x = 0, y = 0;
    CT m_r = 0, m_i = 0, b = 0;
    if (live) {
        p = sel_pix[c];
        x = p / size;
        y = p - x * size;
        m_r = (CT)model[p].x;
        m_i = (CT)model[p].y;
        b = (CT)bg[p];
    }
    double nll = 0., gr = 0., gi = 0.;
    for (int k = 0; k < EN_FRAMES; ++k) {
        const long long d = d0 + k;
        if (d >= n_frames) break;
        const CT vs = (CT)(vscale * scale[d]);
        double ga = 0., gd = 0., gx = 0., gy = 0.;
        if (live) {
            const Holo<CT> h = holo_ref<CT>(x, y, size, (CT)dia[d], (CT)sx[d], (CT)sy[d]);
            const CT zr = m_r + h.rr, zi = m_i + h.ri;
            const CT w = zr * zr + zi * zi + b;
            nll += (double)(vs * w);
            if (GRAD) {
                const CT wr = (CT)2 * vs * zr, wi = (CT)2 * vs * zi;   // d(vs W)/dz
                gr += (double)wr;
                gi += (double)wi;
                ga = vscale * (double)w;
                gd = (double)(wr * h.dd_r + wi * h.dd_i);
                gx = (double)(wr * h.dx_r + wi * h.dx_i);
                gy = (double)(wr * h.dy_r + wi * h.dy_i);
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
            atomicAdd(&gre[p], gr);
            atomicAdd(&gim[p], gi);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < EN_FRAMES; i += blockDim.x) {
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

// Photon term: one warp per frame, lanes over its photons on likelihood
// pixels.  Each photon's rotated position and bilinear weights follow
// rot_log_value exactly (same operations), the four corners' W are
// recomputed, and the adjoint goes back to those corners.
template <typename CT, bool GRAD>
__global__ void __launch_bounds__(256)
k_emc_nll_photons(const int *__restrict__ ones, const int *__restrict__ multi,
                  const long long *__restrict__ ones_accum,
                  const long long *__restrict__ multi_accum, const int *__restrict__ place_ones,
                  const int *__restrict__ place_multi, const int *__restrict__ count_multi,
                  long long n_frames, const double2 *__restrict__ model, int size,
                  const double *__restrict__ bg, const int *__restrict__ pix2sel,
                  const double *__restrict__ rot_cs, const double *__restrict__ dia,
                  const double *__restrict__ sx, const double *__restrict__ sy,
                  const double *__restrict__ scale, double *__restrict__ out,
                  double *__restrict__ gre, double *__restrict__ gim, double *__restrict__ gdia,
                  double *__restrict__ gsx, double *__restrict__ gsy,
                  double *__restrict__ gscale, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long npix = (long long)size * size;
    const int cen = size / 2;
    double nll = 0.;
    for (long long d = warp; d < n_frames; d += nwarp) {
        const double ac = rot_cs[2 * d], as = rot_cs[2 * d + 1];
        const double sd = scale[d];
        const CT dd = (CT)dia[d], xd = (CT)sx[d], yd = (CT)sy[d];
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
            if (pix2sel[p] < 0 || cnt <= 0) continue;
            const double k = (double)cnt;
            nll -= k * log(sd);
            if (GRAD) ga -= k / sd;
            const int x = p / size, y = p - (p / size) * size;
            const double xc = (double)(x - cen), yc = (double)(y - cen);
            const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
            const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
            const double fxl = floor(tx), fyl = floor(ty);
            if (fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2) {
                nll += 1000. * k;                   // L = -1000, no gradient
                continue;
            }
            const int ix = (int)fxl, iy = (int)fyl;
            const double fx = tx - fxl, fy = ty - fyl;
            const double cx = 1. - fx, cy = 1. - fy;
            // corners in rot_log_value's order: (ix, iy), (ix + 1, iy),
            // (ix, iy + 1), (ix + 1, iy + 1)
            const int qx[4] = {ix, ix + 1, ix, ix + 1};
            const int qy[4] = {iy, iy, iy + 1, iy + 1};
            const double wt[4] = {xmul(cx, cy), xmul(fx, cy), xmul(cx, fy), xmul(fx, fy)};
            CT zr[4], zi[4];
            Holo<CT> h[4];
            double v = 0.;
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const long long q = (long long)qx[c4] * size + qy[c4];
                h[c4] = holo_ref<CT>(qx[c4], qy[c4], size, dd, xd, yd);
                zr[c4] = (CT)model[q].x + h[c4].rr;
                zi[c4] = (CT)model[q].y + h[c4].ri;
                const double w = (double)(zr[c4] * zr[c4] + zi[c4] * zi[c4]) + bg[q];
                v += wt[c4] * w;
            }
            v += bg[p];
            if (v < 1.e-20) {
                nll += 1000. * k;
                continue;
            }
            nll -= k * log(v);
            if (GRAD) {
                const double g = -k / v;
#pragma unroll
                for (int c4 = 0; c4 < 4; ++c4) {
                    const long long q = (long long)qx[c4] * size + qy[c4];
                    const CT gc = (CT)(g * wt[c4]);
                    const CT wr = (CT)2 * gc * zr[c4], wi = (CT)2 * gc * zi[c4];
                    atomicAdd(&gre[q], (double)wr);
                    atomicAdd(&gim[q], (double)wi);
                    gd += (double)(wr * h[c4].dd_r + wi * h[c4].dd_i);
                    gx += (double)(wr * h[c4].dx_r + wi * h[c4].dx_i);
                    gy += (double)(wr * h[c4].dy_r + wi * h[c4].dy_i);
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
void emc_launch(const double2 *model, int size, const double *bg, const int *sel_pix,
                long long n_sel, const int *pix2sel, const int *ones, const int *multi,
                const long long *oacc, const long long *macc, const int *po, const int *pm,
                const int *cm, long long n_frames, const double *rot_cs, const double *dia,
                const double *sx, const double *sy, const double *scale, double vscale,
                double *out, double *gre, double *gim, double *gdia, double *gsx, double *gsy,
                double *gscale, int *err, cudaStream_t stream) {
    if (n_sel > 0) {
        const dim3 grid((unsigned)((n_sel + 255) / 256),
                        (unsigned)((n_frames + EN_FRAMES - 1) / EN_FRAMES));
        k_emc_nll_msum<CT, GRAD><<<grid, 256, 0, stream>>>(model, size, bg, sel_pix, n_sel, dia,
                                                           sx, sy, scale, n_frames, vscale, out,
                                                           gre, gim, gdia, gsx, gsy, gscale);
    }
    k_emc_nll_photons<CT, GRAD><<<rspi_blocks(n_frames * 32, 256), 256, 0, stream>>>(
        ones, multi, oacc, macc, po, pm, cm, n_frames, model, size, bg, pix2sel, rot_cs, dia, sx,
        sy, scale, out, gre, gim, gdia, gsx, gsy, gscale, err);
}

}  // namespace

extern "C" int rspi_emc_nll(int precision, int want_grad, const double *model, long long size,
                            const double *bg, const int *sel_pix, long long n_sel,
                            const int *pix2sel, const int *ones, const int *multi,
                            const long long *ones_accum, const long long *multi_accum,
                            const int *place_ones, const int *place_multi,
                            const int *count_multi, long long n_frames, const double *rot_cs,
                            const double *dia, const double *sx, const double *sy,
                            const double *scale, double vscale, double *nll, double *gre,
                            double *gim, double *gdia, double *gsx, double *gsy, double *gscale,
                            int *err, cudaStream_t stream) {
    if (n_frames <= 0 || n_frames > 0xffffLL * EN_FRAMES || size <= 1 || size > 46340 ||
        n_sel < 0 || (n_sel > 0 && !sel_pix) || !model || !bg || !pix2sel || !ones || !multi ||
        !ones_accum || !multi_accum || !rot_cs || !dia || !sx || !sy || !scale || !nll ||
        (precision != 0 && precision != 1))
        return RSPI_ERR_ARG;
    if (want_grad && (!gre || !gim || !gdia || !gsx || !gsy || !gscale)) return RSPI_ERR_ARG;
    const long long npix = size * size;
    cudaMemsetAsync(nll, 0, sizeof(double), stream);
    if (want_grad) {
        cudaMemsetAsync(gre, 0, sizeof(double) * npix, stream);
        cudaMemsetAsync(gim, 0, sizeof(double) * npix, stream);
        cudaMemsetAsync(gdia, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gsx, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gsy, 0, sizeof(double) * n_frames, stream);
        cudaMemsetAsync(gscale, 0, sizeof(double) * n_frames, stream);
    }
    const double2 *m = reinterpret_cast<const double2 *>(model);
#define RSPI_ENLL(CT, G)                                                                       \
    emc_launch<CT, G>(m, (int)size, bg, sel_pix, n_sel, pix2sel, ones, multi, ones_accum,       \
                      multi_accum, place_ones, place_multi, count_multi, n_frames, rot_cs, dia, \
                      sx, sy, scale, vscale, nll, gre, gim, gdia, gsx, gsy, gscale, err, stream)
    if (precision == 1 && want_grad) RSPI_ENLL(double, true);
    else if (precision == 1) RSPI_ENLL(double, false);
    else if (want_grad) RSPI_ENLL(float, true);
    else RSPI_ENLL(float, false);
#undef RSPI_ENLL
    RSPI_RETURN_LAUNCH();
}
