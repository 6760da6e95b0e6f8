// Data simulator (make_data.py:199-333): the reference's per-frame Python
// loop -- frame model, holographic intensity, detector mask, normalisation
// to the mean photon count, in-plane rotation, background, Poisson counts and
// the sparse photon lists -- as four batched kernels over B frames at a time.
//
//   k_sim_view      one CTA per frame: the frame's model (object type iso /
//                   homo / mix / blur, make_data.py:294-309), its holographic
//                   intensity with the frame's sphere shift, diameter,
//                   rel_scale and fluence scale (kernels.cu:44-82 with bg 0),
//                   times the mask, then scaled so that it sums to
//                   mean_count (make_data.py:310-318)
//   k_sim_counts    per (pixel block, frame): the view rotated by the frame's
//                   angle (its cosine and sine from the host) with slice_gen's
//                   bilinear rule (kernels.cu:6-42,
//                   log_flag 0: pixels whose footprint leaves the detector are
//                   0 and get no background), plus bg, then a Poisson draw
//                   (make_data.py:319-323)
//   k_sim_sparse_*  per frame: the number of pixels with one and with several
//                   photons, then those pixels in ascending order with the
//                   counts of the latter (make_data.py:324-328)
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011), counter (pixel, frame low,
// frame high, draw), key = the 64-bit seed, so a frame's counts depend only
// on (seed, frame index, pixel) and not on the batching.  Poisson draws:
// inversion by sequential search below a mean of 10, above it the
// transformed rejection PTRS of Hoermann ("The transformed rejection method
// for generating Poisson random variables", Insurance: Mathematics and
// Economics 12, 1993), both exact samplers of the Poisson law.
#include "rspi_common.cuh"

namespace {

constexpr int SIM_THREADS = 512;
constexpr int FILL_THREADS = 256;
constexpr double PI = 3.14159265358979311599796346854;  // the double nearest pi
constexpr int PTRS_MAX_TRIES = 512;   // rejection rounds (acceptance is above 85% per round)

struct U4 {
    unsigned x, y, z, w;
};

// Philox4x32 with 10 rounds; multipliers and key increments of the paper.
__device__ __forceinline__ U4 philox(U4 c, unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Uniform double in (0, 1) from 53 of 64 random bits (never 0 or 1).
__device__ __forceinline__ double unit_open(unsigned hi, unsigned lo) {
    const unsigned long long b = (((unsigned long long)hi << 32) | lo) >> 11;
    return ((double)b + 0.5) * 0x1.0p-53;
}

struct Stream {
    unsigned pix, flo, fhi, k0, k1, draw;
    __device__ U4 next() { return philox(U4{pix, flo, fhi, draw++}, k0, k1); }
};

// One Poisson(lam) draw; lam must be finite and >= 0 (else *err).
__device__ int poisson_draw(double lam, Stream &st, int *err) {
    if (!(lam >= 0.) || isinf(lam) || lam > 1.e9) {
        rspi_flag(err, RSPI_ERR_ARG);
        return 0;
    }
    if (lam == 0.) return 0;
    if (lam < 10.) {
        const U4 r = st.next();
        const double u = unit_open(r.x, r.y);
        double p = exp(-lam), cdf = p;
        int k = 0;
        while (u > cdf && p > 0. && k < 4096) {
            ++k;
            p = p * lam / (double)k;
            cdf += p;
        }
        return k;
    }
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.);
    for (int it = 0; it < PTRS_MAX_TRIES; ++it) {
        const U4 r = st.next();
        const double u = unit_open(r.x, r.y) - 0.5;
        const double v = unit_open(r.z, r.w);
        const double us = 0.5 - fabs(u);
        const double k = floor((2. * a / us + b) * u + lam + 0.43);
        if (us >= 0.07 && v <= vr) return (int)k;
        if (k < 0. || (us < 0.013 && v > us)) continue;
        if (log(v) + log(inv_alpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.))
            return (int)k;
    }
    rspi_flag(err, RSPI_ERR_TIMEOUT);
    return (int)floor(lam + 0.5);
}

// The frame's Fourier model at pixel (x, y) (make_data.py:294-309).  kind: 0
// iso, 1 homo, 2 mix, 3 blur; w the frame's wobble amplitude; ramps
// e^{2 pi i (qx w + qy w)} ("A") and e^{2 pi i (qx w - 3.7 qy w)} ("B") with
// qx = (x - c) / 2c, qy = (y - c) / 2c, c = size // 2; np.fliplr takes column
// size - 1 - y.
__device__ __forceinline__ double2 ramp_term(const double2 *wob, int x, int y, int size,
                                             double w, bool b_ramp) {
    const double c = (double)(size / 2);
    const double qx = ((double)x - c) / (2. * c), qy = ((double)y - c) / (2. * c);
    const double arg = b_ramp ? xadd(xmul(qx, w), xmul(xmul(-3.7, qy), w))
                              : xadd(xmul(qx, w), xmul(qy, w));
    double s, co;
    sincos(xmul(2. * PI, arg), &s, &co);
    const double2 m = wob[(long long)x * size + y];
    return make_double2(xsub(xmul(m.x, co), xmul(m.y, s)), xadd(xmul(m.x, s), xmul(m.y, co)));
}

__device__ __forceinline__ double2 frame_model(const double2 *model, const double2 *wob, int kind,
                                               long long frame, double w, int x, int y,
                                               int size) {
    double2 f = model[(long long)x * size + y];
    if (kind == 0) return f;
    const int yf = size - 1 - y;
    double2 t;
    if (kind == 1) {
        const double2 a = ramp_term(wob, x, yf, size, w, true);
        const double2 b = ramp_term(wob, x, y, size, w, false);
        t = make_double2(xadd(a.x, b.x) / 2., xadd(a.y, b.y) / 2.);
    } else if (kind == 2) {
        t = (frame & 1) == 0 ? ramp_term(wob, x, y, size, w, false)
                             : ramp_term(wob, x, yf, size, w, true);
    } else {
        t = ramp_term(wob, x, y, size, w, true);
    }
    return make_double2(xadd(f.x, t.x), xadd(f.y, t.y));
}

__global__ void __launch_bounds__(SIM_THREADS)
k_sim_view(const double2 *__restrict__ model, const double2 *__restrict__ wob, int kind,
           long long frame0, const double *__restrict__ wobble, const double *__restrict__ shifts,
           const double *__restrict__ dia, const double *__restrict__ scale, double rel_scale,
           double mean_count, double mask_value, int size, double *__restrict__ view,
           int *__restrict__ err) {
    __shared__ double scratch[32];
    const long long f = blockIdx.x;
    const long long npix = (long long)size * size;
    const double sx = shifts[2 * f], sy = shifts[2 * f + 1], d = dia[f], sc = scale[f];
    const double w = wobble ? wobble[f] : 0.;
    const double cen = floor(size / 2.), dsize = (double)size;
    const int icen = size / 2;
    double *v = view + f * npix;
    double acc = 0.;
    for (long long p = threadIdx.x; p < npix; p += blockDim.x) {
        const int x = (int)(p / size), y = (int)(p - (long long)x * size);
        const double dx = (double)x - cen, dy = (double)y - cen;
        // detector mask (make_data.py:210-216): r < 4 or r >= size // 2 is 0
        const double r = sqrt(xadd(xmul((double)(x - icen), (double)(x - icen)),
                                   xmul((double)(y - icen), (double)(y - icen))));
        double val = 0.;
        if (!(r < 4.) && !(r >= (double)icen)) {
            const double2 m = frame_model(model, wob, kind, frame0 + f, w, x, y, size);
            const double phase = xmul(2. * PI, xadd(xmul(dx, sx), xmul(dy, sy))) / dsize;
            double s = xmul(xmul(sqrt(xadd(xmul(dx, dx), xmul(dy, dy))), PI), d) / dsize;
            if (s == 0.) s = 1.e-5;
            const double sphere = xmul(rel_scale, xsub(sin(s), xmul(s, cos(s)))) / xmul(xmul(s, s), s);
            const double re = xadd(xmul(cos(phase), sphere), m.x);
            const double im = xadd(xmul(sin(phase), sphere), m.y);
            val = xmul(xmul(xadd(xmul(re, re), xmul(im, im)), sc), mask_value);
        }
        v[p] = val;
        acc += val;
    }
    const double total = block_sum(acc, scratch);
    if (!(total > 0.) || isinf(total)) {
        if (threadIdx.x == 0) rspi_flag(err, RSPI_ERR_ARG);
        return;
    }
    const double factor = mean_count / total;
    for (long long p = threadIdx.x; p < npix; p += blockDim.x) v[p] = xmul(v[p], factor);
}

__global__ void k_sim_counts(const double *__restrict__ view, long long frame0,
                             const double *__restrict__ rot_cs, const double *__restrict__ bg,
                             int size, unsigned k0, unsigned k1, int *__restrict__ counts,
                             double *__restrict__ expected, int *__restrict__ err) {
    const long long f = blockIdx.y;
    const long long npix = (long long)size * size;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    const double *v = view + f * npix;
    const int x = (int)(p / size), y = (int)(p - (long long)x * size);
    const int cen = size / 2;
    const double ac = rot_cs[2 * f], as = rot_cs[2 * f + 1];
    const double xc = (double)(x - cen), yc = (double)(y - cen);
    const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
    const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
    const double fxl = floor(tx), fyl = floor(ty);
    double lam = 0.;
    if (!(fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2)) {
        const int ix = (int)fxl, iy = (int)fyl;
        const double fx = xsub(tx, fxl), fy = xsub(ty, fyl);
        const double cx = xsub(1., fx), cy = xsub(1., fy);
        const long long b0 = (long long)ix * size + iy;
        lam = xadd(xadd(xadd(xmul(xmul(v[b0], cx), cy), xmul(xmul(v[b0 + size], fx), cy)),
                        xmul(xmul(v[b0 + 1], cx), fy)),
                   xmul(xmul(v[b0 + size + 1], fx), fy));
        if (bg) lam = xadd(lam, bg[p]);
    }
    if (expected) expected[f * npix + p] = lam;
    const unsigned long long fg = (unsigned long long)(frame0 + f);
    Stream st{(unsigned)p, (unsigned)fg, (unsigned)(fg >> 32), k0, k1, 0u};
    counts[f * npix + p] = poisson_draw(lam, st, err);
}

__global__ void k_sim_poisson(const double *__restrict__ lam, long long n, unsigned k0,
                              unsigned k1, unsigned long long stream_id, int *__restrict__ out,
                              int *__restrict__ err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Stream st{(unsigned)i, (unsigned)(i >> 32) ^ (unsigned)stream_id,
                  (unsigned)(stream_id >> 32) ^ 0x80000000u, k0, k1, 0u};
        out[i] = poisson_draw(lam[i], st, err);
    }
}

__global__ void __launch_bounds__(FILL_THREADS)
k_sim_sparse_counts(const int *__restrict__ counts, long long npix, int *__restrict__ ones,
                    int *__restrict__ multi) {
    __shared__ int s1[FILL_THREADS / 32], sm[FILL_THREADS / 32];
    const long long f = blockIdx.x;
    const int *c = counts + f * npix;
    int n1 = 0, nm = 0;
    for (long long p = threadIdx.x; p < npix; p += blockDim.x) {
        const int v = c[p];
        n1 += v == 1;
        nm += v > 1;
    }
    n1 = warp_sum(n1);
    nm = warp_sum(nm);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s1[wid] = n1;
        sm[wid] = nm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0;
        for (int k = 0; k < FILL_THREADS / 32; ++k) {
            a += s1[k];
            b += sm[k];
        }
        ones[f] = a;
        multi[f] = b;
    }
}

// Pixels with one photon, and with several (and their counts), in ascending
// order: blockDim pixels at a time, ranks from warp ballots and the warps'
// totals before them.
__global__ void __launch_bounds__(FILL_THREADS)
k_sim_sparse_fill(const int *__restrict__ counts, long long npix,
                  const long long *__restrict__ ones_off, const long long *__restrict__ multi_off,
                  int *__restrict__ place_ones, int *__restrict__ place_multi,
                  int *__restrict__ count_multi) {
    constexpr int NW = FILL_THREADS / 32;
    __shared__ int w1[NW], wm[NW];
    const long long f = blockIdx.x;
    const int *c = counts + f * npix;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    long long o1 = ones_off[f], om = multi_off[f];
    for (long long base = 0; base < npix; base += FILL_THREADS) {
        const long long p = base + threadIdx.x;
        const int v = p < npix ? c[p] : 0;
        const unsigned b1 = __ballot_sync(RSPI_FULL_MASK, v == 1);
        const unsigned bm = __ballot_sync(RSPI_FULL_MASK, v > 1);
        if (lane == 0) {
            w1[wid] = __popc(b1);
            wm[wid] = __popc(bm);
        }
        __syncthreads();
        long long before1 = 0, beforem = 0, tot1 = 0, totm = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            if (k < wid) {
                before1 += w1[k];
                beforem += wm[k];
            }
            tot1 += w1[k];
            totm += wm[k];
        }
        if (v == 1) place_ones[o1 + before1 + __popc(b1 & below)] = (int)p;
        if (v > 1) {
            const long long q = om + beforem + __popc(bm & below);
            place_multi[q] = (int)p;
            count_multi[q] = v;
        }
        o1 += tot1;
        om += totm;
        __syncthreads();
    }
}

}  // namespace

extern "C" int rspi_sim_views(const double *model, const double *wobble_model, int kind,
                              long long frame0, long long n_frames, const double *wobble,
                              const double *shifts, const double *dia, const double *scale,
                              double rel_scale, double mean_count, double mask_value, int size,
                              double *view, int *err, cudaStream_t stream) {
    if (!model || !shifts || !dia || !scale || !view || !err || n_frames <= 0 ||
        n_frames > 0x7fffffffLL || frame0 < 0 || size < 2 || size > 46340 || kind < 0 ||
        kind > 3 || (kind != 0 && (!wobble_model || !wobble)))
        return RSPI_ERR_ARG;
    k_sim_view<<<(unsigned)n_frames, SIM_THREADS, 0, stream>>>(
        reinterpret_cast<const double2 *>(model), reinterpret_cast<const double2 *>(wobble_model),
        kind, frame0, wobble, shifts, dia, scale, rel_scale, mean_count, mask_value, size, view,
        err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sim_counts(const double *view, long long frame0, long long n_frames,
                               const double *rot_cs, const double *bg, int size,
                               unsigned long long seed, int *counts, double *expected, int *err,
                               cudaStream_t stream) {
    if (!view || !rot_cs || !counts || !err || n_frames <= 0 || n_frames > 65535 || frame0 < 0 ||
        size < 2 || size > 46340)
        return RSPI_ERR_ARG;
    const long long npix = (long long)size * size;
    const dim3 grid((unsigned)((npix + 255) / 256), (unsigned)n_frames);
    k_sim_counts<<<grid, 256, 0, stream>>>(view, frame0, rot_cs, bg, size, (unsigned)seed,
                                           (unsigned)(seed >> 32), counts, expected, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sim_poisson(const double *lam, long long n, unsigned long long seed,
                                unsigned long long stream_id, int *out, int *err,
                                cudaStream_t stream) {
    if (!lam || !out || !err || n <= 0 || n > 0xffffffffLL) return RSPI_ERR_ARG;
    k_sim_poisson<<<rspi_blocks(n, 256), 256, 0, stream>>>(lam, n, (unsigned)seed,
                                                          (unsigned)(seed >> 32), stream_id,
                                                          out, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sim_sparse_counts(const int *counts, long long n_frames, long long num_pix,
                                      int *ones, int *multi, cudaStream_t stream) {
    if (!counts || !ones || !multi || n_frames <= 0 || n_frames > 0x7fffffffLL ||
        num_pix <= 0 || num_pix > 0x7fffffffLL)
        return RSPI_ERR_ARG;
    k_sim_sparse_counts<<<(unsigned)n_frames, FILL_THREADS, 0, stream>>>(counts, num_pix, ones,
                                                                       multi);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sim_sparse_fill(const int *counts, long long n_frames, long long num_pix,
                                    const long long *ones_off, const long long *multi_off,
                                    int *place_ones, int *place_multi, int *count_multi,
                                    cudaStream_t stream) {
    if (!counts || !ones_off || !multi_off || !place_ones || !place_multi || !count_multi ||
        n_frames <= 0 || n_frames > 0x7fffffffLL || num_pix <= 0 || num_pix > 0x7fffffffLL)
        return RSPI_ERR_ARG;
    k_sim_sparse_fill<<<(unsigned)n_frames, FILL_THREADS, 0, stream>>>(
        counts, num_pix, ones_off, multi_off, place_ones, place_multi, count_multi);
    RSPI_RETURN_LAUNCH();
}
