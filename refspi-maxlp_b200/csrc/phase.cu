// Model refinement after the pattern search: error reduction and the
// difference map (maxLP.py:271-298, 342-354), on the device.
//
// The reference transforms with NumPy's centred convention
// fftshift(fftn(ifftshift(x))) and its inverse.  For a line of n values and
// c = n / 2 that is
//     y[k] = sum_j x[j] * exp(s * 2 pi i (j - c)(k - c) / n),  s = -1 (+1 and
//     a factor 1/n for the inverse),
// a DFT whose phase index (j - c)(k - c) is reduced mod n exactly in integer
// arithmetic, so every term uses one entry of an n-entry twiddle table.  Model
// images are at most a few hundred pixels a side: a line transform of n
// outputs of n terms each (FP64, complex FMA) costs about what the host's
// FFT costs per image and keeps the FP64 error near n * 2^-53 of the line's
// magnitude.  A 2-D transform is a pass over the rows (contiguous) and one
// over the columns; the column pass carries the projection arithmetic that
// follows it in its epilogue.
//
// Support (maxLP.py:292-298): fconv tapered by expit((mrad - 12) / 2), the
// centred inverse transform, |real part| smoothed by a Gaussian (sigma 3,
// radius 12 = int(4 sigma + 0.5), 'reflect' edges: d c b a | a b c d, axis 0
// then axis 1, the symmetric-kernel order w0 x0 + sum over k = radius..1 of
// wk (x-k + x+k)), then
// thresholded: minvsupp = !(smoothed > 1.2e-4).
#include "rspi_common.cuh"

namespace {

constexpr int MAX_N = 1024;          // longest line a CTA transforms
constexpr int MAX_RADIUS = 64;       // longest Gaussian half-width

// Epilogues of the column pass (one output element each).
enum Epilogue : int {
    EP_STORE = 0,        // y
    EP_REAL_PROJ = 1,    // (max(re y, 0), 0), 0 outside the support
    EP_DIFFMAP = 2,      // x + y - p1 written over x
    EP_ABS_REAL = 3,     // |re y| into a real array
};

// One CTA per line of the n x n complex image: axis 1 = rows (contiguous),
// axis 0 = columns.  Line transform with the centred phase index, times
// `scale`, then the epilogue.
template <int EP>
__global__ void __launch_bounds__(256)
k_cdft_lines(const double2 *__restrict__ in, double2 *__restrict__ out, int n, int axis,
             int sign, double scale, const unsigned char *__restrict__ minvsupp,
             double2 *__restrict__ x, const double2 *__restrict__ p1, double *__restrict__ out_re) {
    __shared__ double2 line[MAX_N];
    __shared__ double2 tw[MAX_N];
    const int li = blockIdx.x;                      // line index
    const long long stride = axis == 1 ? 1 : n;
    const long long base = axis == 1 ? (long long)li * n : li;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        line[j] = in[base + j * stride];
        double s, c;
        sincospi(2.0 * (double)j / (double)n, &s, &c);
        tw[j] = make_double2(c, sign * s);
    }
    __syncthreads();
    const int cen = n / 2;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int a = ((k - cen) % n + n) % n;      // (k - c) mod n
        int m = (int)(((long long)(n - cen) % n * a) % n);   // (0 - c)(k - c) mod n
        double re = 0., im = 0.;
        for (int j = 0; j < n; ++j) {
            const double2 v = line[j], w = tw[m];
            re = fma(v.x, w.x, re);
            re = fma(-v.y, w.y, re);
            im = fma(v.x, w.y, im);
            im = fma(v.y, w.x, im);
            m += a;
            if (m >= n) m -= n;
        }
        re *= scale;
        im *= scale;
        const long long t = base + k * stride;
        if (EP == EP_STORE) {
            out[t] = make_double2(re, im);
        } else if (EP == EP_REAL_PROJ) {
            const double r = (re < 0. || minvsupp[t]) ? 0. : re;
            out[t] = make_double2(r, 0.);
        } else if (EP == EP_DIFFMAP) {
            const double2 xv = x[t], pv = p1[t];
            x[t] = make_double2(xv.x + re - pv.x, xv.y + im - pv.y);
        } else {
            out_re[t] = fabs(re);
        }
    }
}

// p1 = proj_fourier(fconv, x) (data pixels from fconv); with `dm`, also
// z = 2 p1 - x, the difference map's input to the real-space projection.
__global__ void k_proj_fourier(const double2 *__restrict__ fconv,
                               const unsigned char *__restrict__ minvmask,
                               const double2 *__restrict__ x, double2 *__restrict__ p1,
                               double2 *__restrict__ z, long long npix) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < npix; t += stride) {
        const double2 xv = x[t];
        const double2 p = minvmask[t] ? fconv[t] : xv;
        if (p1) p1[t] = p;
        if (z) z[t] = make_double2(2. * p.x - xv.x, 2. * p.y - xv.y);
    }
}

// fconv * expit((mrad - r0) * slope), mrad the integer-centred radius.
__global__ void k_support_taper(const double2 *__restrict__ fconv, int n, double r0,
                                double slope, double2 *__restrict__ out) {
    const long long npix = (long long)n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cen = n / 2;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < npix; t += stride) {
        const long long xi = t / n, yi = t - xi * n;
        const double dx = (double)(xi - cen), dy = (double)(yi - cen);
        const double r = sqrt(dx * dx + dy * dy);
        const double e = 1. / (1. + exp(-((r - r0) * slope)));
        const double2 v = fconv[t];
        out[t] = make_double2(v.x * e, v.y * e);
    }
}

// One CTA per line: correlate with the normalised Gaussian of half-width
// `radius` ('reflect' edges); with `thr_out`, minvsupp = !(value > thr).
__global__ void __launch_bounds__(256)
k_gauss_lines(const double *__restrict__ in, double *__restrict__ out, int n, int axis,
              double sigma, int radius, double thr, unsigned char *__restrict__ minvsupp) {
    __shared__ double line[MAX_N];
    __shared__ double w[MAX_RADIUS + 1];
    const int li = blockIdx.x;
    const long long stride = axis == 1 ? 1 : n;
    const long long base = axis == 1 ? (long long)li * n : li;
    for (int j = threadIdx.x; j < n; j += blockDim.x) line[j] = in[base + j * stride];
    if (threadIdx.x == 0) {
        // phi(x) = exp(-x^2 / (2 sigma^2)) / sum over |x| <= radius
        double sum = 0.;
        for (int k = -radius; k <= radius; ++k) sum += exp(-0.5 / (sigma * sigma) * (double)(k * k));
        for (int k = 0; k <= radius; ++k) w[k] = exp(-0.5 / (sigma * sigma) * (double)(k * k)) / sum;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double acc = line[i] * w[0];
        for (int k = radius; k >= 1; --k) {   // outermost pair first
            int lo = i - k, hi = i + k;
            // reflect about the edge: -1 -> 0, n -> n - 1 (radius < n)
            lo = lo < 0 ? -lo - 1 : lo;
            hi = hi >= n ? 2 * n - hi - 1 : hi;
            acc += (line[lo] + line[hi]) * w[k];
        }
        const long long t = base + i * stride;
        if (minvsupp)
            minvsupp[t] = !(acc > thr);
        else
            out[t] = acc;
    }
}

template <int EP>
void col_pass(const double2 *in, double2 *out, int n, int sign, double scale,
              const unsigned char *minvsupp, double2 *x, const double2 *p1, double *out_re,
              cudaStream_t stream) {
    k_cdft_lines<EP><<<n, 256, 0, stream>>>(in, out, n, 0, sign, scale, minvsupp, x, p1,
                                            out_re);
}

// proj_real(z) = centred forward transform of the clamped, support-masked
// real part of the centred inverse transform of z; the result goes through
// the epilogue EP (store into `out`, or the difference-map combination).
template <int EP>
void proj_real(const double2 *z, const unsigned char *minvsupp, double2 *t1, double2 *t2,
               double2 *out, double2 *x, const double2 *p1, int n, cudaStream_t stream) {
    const double inv_n = 1. / (double)n;
    k_cdft_lines<EP_STORE><<<n, 256, 0, stream>>>(z, t1, n, 1, 1, inv_n, nullptr, nullptr,
                                                  nullptr, nullptr);
    col_pass<EP_REAL_PROJ>(t1, t2, n, 1, inv_n, minvsupp, nullptr, nullptr, nullptr, stream);
    k_cdft_lines<EP_STORE><<<n, 256, 0, stream>>>(t2, t1, n, 1, -1, 1., nullptr, nullptr,
                                                  nullptr, nullptr);
    col_pass<EP>(t1, out, n, -1, 1., nullptr, x, p1, nullptr, stream);
}

bool size_ok(long long n) { return n >= 2 && n <= MAX_N; }

}  // namespace

extern "C" int rspi_cdft2(const double *in, double *out, double *work, long long size,
                          int inverse, cudaStream_t stream) {
    if (!in || !out || !work || !size_ok(size) || (inverse != 0 && inverse != 1))
        return RSPI_ERR_ARG;
    const int n = (int)size;
    const int sign = inverse ? 1 : -1;
    const double scale = inverse ? 1. / (double)n : 1.;
    k_cdft_lines<EP_STORE><<<n, 256, 0, stream>>>(
        reinterpret_cast<const double2 *>(in), reinterpret_cast<double2 *>(work), n, 1, sign,
        scale, nullptr, nullptr, nullptr, nullptr);
    col_pass<EP_STORE>(reinterpret_cast<const double2 *>(work), reinterpret_cast<double2 *>(out),
                       n, sign, scale, nullptr, nullptr, nullptr, nullptr, stream);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_phase_support(const double *fconv, long long size, double taper_radius,
                                  double taper_slope, double sigma, int radius, double threshold,
                                  unsigned char *minvsupp, double *work, cudaStream_t stream) {
    if (!fconv || !minvsupp || !work || !size_ok(size) || radius < 0 || radius > MAX_RADIUS ||
        radius >= size || !(sigma > 0.))
        return RSPI_ERR_ARG;
    const int n = (int)size;
    const long long npix = size * size;
    double2 *t1 = reinterpret_cast<double2 *>(work);
    double2 *t2 = t1 + npix;
    double *re = reinterpret_cast<double *>(t2 + npix);
    double *sm = re + npix;
    const double inv_n = 1. / (double)n;
    k_support_taper<<<rspi_blocks(npix, 256), 256, 0, stream>>>(
        reinterpret_cast<const double2 *>(fconv), n, taper_radius, taper_slope, t1);
    k_cdft_lines<EP_STORE><<<n, 256, 0, stream>>>(t1, t2, n, 1, 1, inv_n, nullptr, nullptr,
                                                  nullptr, nullptr);
    col_pass<EP_ABS_REAL>(t2, nullptr, n, 1, inv_n, nullptr, nullptr, nullptr, re, stream);
    k_gauss_lines<<<n, 256, 0, stream>>>(re, sm, n, 0, sigma, radius, 0., nullptr);
    k_gauss_lines<<<n, 256, 0, stream>>>(sm, nullptr, n, 1, sigma, radius, threshold, minvsupp);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_phase_refine(const double *fconv, const unsigned char *minvmask,
                                 const unsigned char *minvsupp, double *x, double *work,
                                 long long size, int n_dm, int n_er, cudaStream_t stream) {
    if (!fconv || !minvmask || !minvsupp || !x || !work || !size_ok(size) || n_dm < 0 ||
        n_er < 0)
        return RSPI_ERR_ARG;
    const int n = (int)size;
    const long long npix = size * size;
    const double2 *f = reinterpret_cast<const double2 *>(fconv);
    double2 *xv = reinterpret_cast<double2 *>(x);
    double2 *p1 = reinterpret_cast<double2 *>(work);
    double2 *z = p1 + npix;
    double2 *t1 = z + npix;
    double2 *t2 = t1 + npix;
    const unsigned blocks = rspi_blocks(npix, 256);
    for (int it = 0; it < n_dm; ++it) {
        // x + proj_real(2 p1 - x) - p1, written over x
        k_proj_fourier<<<blocks, 256, 0, stream>>>(f, minvmask, xv, p1, z, npix);
        proj_real<EP_DIFFMAP>(z, minvsupp, t1, t2, nullptr, xv, p1, n, stream);
    }
    for (int it = 0; it < n_er; ++it) {
        // proj_real(proj_fourier(fconv, x))
        k_proj_fourier<<<blocks, 256, 0, stream>>>(f, minvmask, xv, p1, nullptr, npix);
        proj_real<EP_STORE>(p1, minvsupp, t1, t2, xv, nullptr, nullptr, n, stream);
    }
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_phase_proj_fourier(const double *fconv, const unsigned char *minvmask,
                                       const double *x, double *out, long long size,
                                       cudaStream_t stream) {
    if (!fconv || !minvmask || !x || !out || !size_ok(size)) return RSPI_ERR_ARG;
    const long long npix = size * size;
    k_proj_fourier<<<rspi_blocks(npix, 256), 256, 0, stream>>>(
        reinterpret_cast<const double2 *>(fconv), minvmask, reinterpret_cast<const double2 *>(x),
        reinterpret_cast<double2 *>(out), nullptr, npix);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_phase_proj_real(const double *x, const unsigned char *minvsupp, double *out,
                                    double *work, long long size, cudaStream_t stream) {
    if (!x || !minvsupp || !out || !work || !size_ok(size)) return RSPI_ERR_ARG;
    const long long npix = size * size;
    double2 *t1 = reinterpret_cast<double2 *>(work);
    double2 *t2 = t1 + npix;
    proj_real<EP_STORE>(reinterpret_cast<const double2 *>(x), minvsupp, t1, t2,
                        reinterpret_cast<double2 *>(out), nullptr, nullptr, (int)size, stream);
    RSPI_RETURN_LAUNCH();
}
