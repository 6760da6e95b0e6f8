// Model slicing (rows a4, a5, a6): holographic slices of every
// (shift, diameter) state, their masked sums, vscale, and the rotated
// log-slices on the likelihood pixels.  FP64 throughout; the rotated slices
// are stored as float32 or float64.
#include <algorithm>

#include <cuda_fp16.h>

#include "rspi_common.cuh"

namespace {

constexpr int HOLO_THREADS = 256;
constexpr double PI = 3.14159265358979311599796346854;  // the double nearest pi

// W[s0][p] = |M(p) + ff(s)*e^{i phase}|^2 + bg(p)   (kernels.cu:58-75)
// phase = 2 pi ((x-cen) sx + (y-cen) sy) / size,  s = sqrt(r2) pi dia / size.
// Operations follow the source order; |z|^2 is re*re + im*im.
__device__ __forceinline__ double holo_value(const double2 m, double dx, double dy, double sx,
                                             double sy, double dia, double size, double bg) {
    const double phase = xmul(2. * PI, xadd(xmul(dx, sx), xmul(dy, sy))) / size;
    double s = xmul(xmul(sqrt(xadd(xmul(dx, dx), xmul(dy, dy))), PI), dia) / size;
    if (s == 0.) s = 1.e-5;
    const double sphere = (1.0 * xsub(sin(s), xmul(s, cos(s)))) / xmul(xmul(s, s), s);
    const double re = xadd(xmul(cos(phase), sphere), m.x);
    const double im = xadd(xmul(sin(phase), sphere), m.y);
    return xadd(xadd(xmul(re, re), xmul(im, im)), bg);
}

__global__ void __launch_bounds__(HOLO_THREADS)
k_holo(const double2 *__restrict__ model, const double *__restrict__ shiftx,
       const double *__restrict__ shifty, const double *__restrict__ sphere_dia, long long size,
       const double *__restrict__ bg, const int *__restrict__ sel_pix, long long n_sel,
       double *__restrict__ holo, double *__restrict__ msum) {
    __shared__ double scratch[32];
    const long long s0 = blockIdx.x;
    const long long npix = size * size;
    const double sx = shiftx[s0], sy = shifty[s0], dia = sphere_dia[s0];
    const double cen = floor(size / 2.);
    const double dsize = (double)size;
    double *w = holo + s0 * npix;
    for (long long p = threadIdx.x; p < npix; p += blockDim.x) {
        const long long x = p / size, y = p - x * size;
        w[p] = holo_value(model[p], (double)x - cen, (double)y - cen, sx, sy, dia, dsize, bg[p]);
    }
    __syncthreads();
    double acc = 0.;
    for (long long c = threadIdx.x; c < n_sel; c += blockDim.x) acc += w[sel_pix[c]];
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) msum[s0] = acc;
}

// EMC.sphere and EMC.ramp of one state (emc.py:244-254): with integer-centred
// x, y and r = sqrt(x^2 + y^2), s = pi r dia / size (1e-5 where 0),
// sphere = (sin s - s cos s) / s^3 and ramp = e^{2 pi i (x sx + y sy) / size}.
__global__ void k_sphere_ramp(int size, double sx, double sy, double dia,
                              double *__restrict__ sphere, double2 *__restrict__ ramp) {
    const long long npix = (long long)size * size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const double cen = (double)(size / 2), dsize = (double)size;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += stride) {
        const long long xi = p / size, yi = p - xi * size;
        const double x = (double)xi - cen, y = (double)yi - cen;
        if (sphere) {
            double sv = xmul(xmul(PI, sqrt(xadd(xmul(x, x), xmul(y, y)))), dia) / dsize;
            if (sv == 0.) sv = 1.e-5;
            sphere[p] = xsub(sin(sv), xmul(sv, cos(sv))) / pow(sv, 3.);
        }
        if (ramp) {
            const double ph = xmul(2. * PI, xadd(xmul(x, sx), xmul(y, sy))) / dsize;
            ramp[p] = make_double2(cos(ph), sin(ph));
        }
    }
}

// vscale = sum_sel powder / sum_s0 msum * S0 ; init = -(msum * vscale)  (emc.py:181,199)
__global__ void __launch_bounds__(1024)
k_vscale_init(const double *__restrict__ msum, long long n_states0,
              const double *__restrict__ powder, const int *__restrict__ sel_pix, long long n_sel,
              double *__restrict__ vscale, double *__restrict__ init) {
    __shared__ double scratch[32];
    double a = 0., b = 0.;
    for (long long c = threadIdx.x; c < n_sel; c += blockDim.x) a += powder[sel_pix[c]];
    for (long long s = threadIdx.x; s < n_states0; s += blockDim.x) b += msum[s];
    a = block_sum(a, scratch);
    b = block_sum(b, scratch);
    const double vs = a / b * (double)n_states0;
    if (threadIdx.x == 0) *vscale = vs;
    for (long long s = threadIdx.x; s < n_states0; s += blockDim.x) init[s] = -(msum[s] * vs);
}

// Rotated log-slices (row s0 * num_rot + j of every state s0 and rotation
// j; zeros past n_sel), rotation-major: a CTA takes one rotation j and up to
// RL_STATES consecutive states.  The rotated position of each likelihood
// column (pixel row/column, the FP64 rotation, floors and the in-detector
// test) depends on (j, column) only, so it is computed once per column and
// reused for every state; each state then costs its four bilinear loads,
// the same FP64 interpolation and log as rot_log_value (identical values)
// and one store.  With PAIRS the four neighbours come as two 16-byte loads
// from the paired copy hp[p] = (w[p], w[p + 1]) of the holographic slices.
constexpr int RL_STATES = 8;

// hp[i] = (holo[i], holo[i + 1]) over the whole state-major array (0 past
// its end); only pairs of a pixel and its right neighbour in the same row
// are read.
__global__ void k_holo_pairs(const double *__restrict__ holo, long long total,
                             double2 *__restrict__ hp) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
        hp[i] = make_double2(holo[i], i + 1 < total ? holo[i + 1] : 0.);
}

// The four bilinear corners of every pixel rounded to FP32, for the
// frame-set slices' FP32 arithmetic: hq[i] = (W[i], W[i + 1], W[i + size],
// W[i + size + 1]) (zero past the end; corners that wrap into the next row
// or state belong to no in-detector footprint), one 16-byte load per value.
__global__ void k_holo_quads32(const double *__restrict__ holo, long long total, int size,
                               float4 *__restrict__ hq) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        auto at = [&](long long j) { return j < total ? (float)holo[j] : 0.f; };
        hq[i] = make_float4(at(i), at(i + 1), at(i + size), at(i + size + 1));
    }
}

template <typename TL, bool PAIRS>
__global__ void __launch_bounds__(256)
k_rot_log_js(const double *__restrict__ holo, const double2 *__restrict__ hp, int num_rot,
             const double *__restrict__ rot_cs,
             int size, const double *__restrict__ bg, const int *__restrict__ sel_pix, int n_sel,
             int p_pad, long long row_begin, long long row_end, long long s_lo, int n_groups,
             TL *__restrict__ out, float *__restrict__ abs_max) {
    const int j = (int)(blockIdx.x % (unsigned)num_rot);
    const long long s_first = s_lo + (long long)(blockIdx.x / (unsigned)num_rot) * RL_STATES;
    const long long npix = (long long)size * size;
    const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
    const int cen = size / 2;
    const float inv_size = 1.f / (float)size;
    // this CTA's states whose row s0 * num_rot + j lies in [row_begin, row_end)
    long long sb = s_first, se = s_first + RL_STATES;
    while (sb < se && sb * num_rot + j < row_begin) ++sb;
    while (se > sb && (se - 1) * num_rot + j >= row_end) --se;
    float amax = 0.f;
    if (sb < se) {
        for (int c = threadIdx.x; c < p_pad; c += blockDim.x) {
            bool in = false;
            long long base = 0;
            double fx = 0., fy = 0., cx = 0., cy = 0., b = 0.;
            if (c < n_sel) {
                const int p = sel_pix[c];
                int x, y;
                pixel_xy(p, size, inv_size, x, y);
                const double xc = (double)(x - cen), yc = (double)(y - cen);
                const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
                const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
                const double fxl = floor(tx), fyl = floor(ty);
                in = !(fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2);
                if (in) {
                    base = (long long)(int)fxl * size + (int)fyl;
                    fx = tx - fxl;
                    fy = ty - fyl;
                    cx = 1. - fx;
                    cy = 1. - fy;
                }
                b = bg[p];
            }
            for (long long s0 = sb; s0 < se; ++s0) {
                double v = 0.;
                if (c < n_sel) {
                    if (in) {
                        double w00, w01, w10, w11;   // w[ix + a][iy + b] as w_ab
                        if constexpr (PAIRS) {
                            const double2 a = hp[s0 * npix + base], b2 = hp[s0 * npix + base + size];
                            w00 = a.x;
                            w01 = a.y;
                            w10 = b2.x;
                            w11 = b2.y;
                        } else {
                            const double *r0 = holo + s0 * npix + base;
                            w00 = r0[0];
                            w01 = r0[1];
                            w10 = r0[size];
                            w11 = r0[size + 1];
                        }
                        double t = xmul(xmul(w00, cx), cy);
                        t = xadd(t, xmul(xmul(w10, fx), cy));
                        t = xadd(t, xmul(xmul(w01, cx), fy));
                        t = xadd(t, xmul(xmul(w11, fx), fy));
                        t = xadd(t, b);
                        v = t < 1.e-20 ? -1000. : log(t);
                    } else {
                        v = -1000.;
                    }
                }
                const TL q = static_cast<TL>(v);
                out[(s0 * num_rot + j - row_begin) * (long long)p_pad + c] = q;
                amax = fmaxf(amax, fabsf(static_cast<float>(q)));
            }
        }
    }
    if (abs_max) {
        amax = __int_as_float(warp_max_int(__float_as_int(amax)));
        if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(abs_max), __float_as_int(amax));
    }
}

// Rotated log-slices in the layout of the frame-set screening kernel: rows
// taken four at a time from row_begin (tile q = (r - row_begin) / 4, lane
// (r - row_begin) mod 4) and columns cut into n_parts parts of part_w, so
// that one tile's part is one contiguous run of float4 columns:
// out[((q * n_parts + h) * part_w + c') * 4 + lane] holds column
// h * part_w + c' (zero past n_sel).  A CTA takes four consecutive rotations
// j0..j0+3 and up to RL_STATES consecutive states; per column the four
// rotated positions are computed once and reused for every state, and with
// num_rot and row_begin multiples of four a state's four rotations are one
// tile's four rows, stored as one 16-byte write.  Values are those of
// rot_log_value (same operations, identical bits).
//
// k_rot_log_sets computes them in FP64 from the paired copy.
// k_rot_log_sets32 computes the value of each (state, rotation) in FP32
// from an FP32 copy of the four corners: bilinear interpolation of positive
// terms (|relative error| <= 9u, u = 2^-24: the FP32 roundings of W, the
// weights and bg, four products and four sums), then ln t = ln2 lg2(t)
// with lg2.approx.f32 (|error| <= 2^-21 + 2^-22 |lg2|, checked over every
// float of [2^-100, 2^100] by rspi_log2_error_max) and one FP32 product
// by the float nearest ln 2 (2u relative with its own rounding):
// |L32 - L| <= u (9.1 + 8 ln2 + (4 + 2.1) |L|) <= 2^-24 (16 + 7 |L|).  The
// rotated positions, floors and the in-detector test stay FP64, and an
// interpolated value at or below 2e-20 (or above 1e30) is computed in FP64
// instead, so the -1000 sentinel is taken exactly where the reference takes
// it.

// ln t as ln2 * lg2.approx(t) for a normal positive t (the bound above).
__device__ __forceinline__ float ln_fast(float t) {
    float l;
    asm("lg2.approx.f32 %0, %1;" : "=f"(l) : "f"(t));
    return __fmul_rn(0x1.62e430p-1f, l);
}

// FP64 value of one (state, rotation, column) for the FP32 path's rare
// fallback: the operations of the FP64 path (and of rot_log_value), the
// rotated position recomputed from (x, y) so that the FP32 path keeps no
// FP64 geometry live.
__device__ __noinline__ float rot_log_fp64(const double2 *__restrict__ w2, int x, int y,
                                           int size, double ac, double as, double b) {
    const int cen = size / 2;
    const double xc = (double)(x - cen), yc = (double)(y - cen);
    const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
    const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
    const double fxl = floor(tx), fyl = floor(ty);
    if (fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2) return -1000.f;
    const long long base = (long long)fxl * size + (long long)fyl;
    const double fx = tx - fxl, fy = ty - fyl;
    const double2 a = w2[base];
    const double2 b2 = w2[base + size];
    const double cx = 1. - fx, cy = 1. - fy;
    double t = xmul(xmul(a.x, cx), cy);
    t = xadd(t, xmul(xmul(b2.x, fx), cy));
    t = xadd(t, xmul(xmul(a.y, cx), fy));
    t = xadd(t, xmul(xmul(b2.y, fx), fy));
    t = xadd(t, b);
    return (float)(t < 1.e-20 ? -1000. : log(t));
}

// The FP32-arithmetic form of k_rot_log_sets (its values as described
// there): per column only the four rotations' in-detector bits, corner
// indices and FP32 weights stay live across the states, so that 1,024
// threads fit an SM (64 registers), a value's four corners come in one
// 16-byte load of the quad copy, and a state's four loads (one per rotation)
// are all issued before any is used: 4.88 ms instead of 8.17 ms (256
// threads, 108 registers, two 8-byte pair loads, one rotation's load in
// flight at a time) for the 72,900 rows x 24,928 columns of a 185^2
// detector, with identical values.
__global__ void __launch_bounds__(1024, 1)
k_rot_log_sets32(const double2 *__restrict__ hp, const float4 *__restrict__ hq, int num_rot,
                 const double *__restrict__ rot_cs, int size, const double *__restrict__ bg,
                 const int *__restrict__ sel_pix, int n_sel, int n_parts, int part_w,
                 long long row_begin, long long row_end, long long s_lo,
                 float *__restrict__ out, float *__restrict__ abs_max) {
    const int n_jb = (num_rot + 3) / 4;
    const int j0 = (int)(blockIdx.x % (unsigned)n_jb) * 4;
    const long long s_first = s_lo + (long long)(blockIdx.x / (unsigned)n_jb) * RL_STATES;
    const long long npix = (long long)size * size;
    const long long n_rows = row_end - row_begin;
    const int cen = size / 2;
    const float inv_size = 1.f / (float)size;
    long long sb = s_first, se = s_first + RL_STATES;
    while (sb < se && sb * num_rot + min(j0 + 3, num_rot - 1) < row_begin) ++sb;
    while (se > sb && (se - 1) * num_rot + j0 >= row_end) --se;
    const int n_cols = n_parts * part_w;
    float amax = 0.f;
    if (sb < se) {
        for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
            const int h = c / part_w, cl = c - h * part_w;
            unsigned inmask = 0;
            int base[4] = {0, 0, 0, 0};
            float fxf[4] = {0.f, 0.f, 0.f, 0.f}, fyf[4] = {0.f, 0.f, 0.f, 0.f};
            float cxf[4] = {0.f, 0.f, 0.f, 0.f}, cyf[4] = {0.f, 0.f, 0.f, 0.f};
            int x = 0, y = 0;
            double b = 0.;
            const bool real = c < n_sel;
            if (real) {
                const int p = sel_pix[c];
                pixel_xy(p, size, inv_size, x, y);
                const double xc = (double)(x - cen), yc = (double)(y - cen);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j = min(j0 + q, num_rot - 1);
                    const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
                    const double tx = xadd(xsub(xmul(xc, ac), xmul(yc, as)), (double)cen);
                    const double ty = xadd(xadd(xmul(xc, as), xmul(yc, ac)), (double)cen);
                    const double fxl = floor(tx), fyl = floor(ty);
                    const bool in = !(fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2);
                    const double fx = in ? tx - fxl : 0., fy = in ? ty - fyl : 0.;
                    inmask |= (unsigned)in << q;
                    base[q] = in ? (int)fxl * size + (int)fyl : 0;
                    fxf[q] = (float)fx;
                    fyf[q] = (float)fy;
                    cxf[q] = (float)(1. - fx);
                    cyf[q] = (float)(1. - fy);
                }
                b = bg[p];
            }
            const float bf = (float)b;
            for (long long s0 = sb; s0 < se; ++s0) {
                // the four rotations' corner loads first, all in flight at
                // once (an out-of-detector or padding column reads corner 0,
                // a valid address, with zero weights, and ignores it)
                float4 w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) w[q] = hq[s0 * npix + base[q]];   // 00, 01, 10, 11
                float v[4];
                unsigned slow = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float t = w[q].x * cxf[q] * cyf[q];
                    t += w[q].z * fxf[q] * cyf[q];
                    t += w[q].y * cxf[q] * fyf[q];
                    t += w[q].w * fxf[q] * fyf[q];
                    t += bf;
                    const bool in = (inmask >> q) & 1u;
                    const bool ok = t > 2.e-20f && t < 1.e30f;
                    v[q] = !real ? 0.f : !in ? -1000.f : ok ? ln_fast(t) : 0.f;
                    slow |= (unsigned)(real && in && !ok) << q;
                }
                if (slow) {
                    // at or below 2e-20 (or above 1e30): the FP64 value
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!((slow >> q) & 1u)) continue;
                        const int j = min(j0 + q, num_rot - 1);
                        v[q] = rot_log_fp64(hp + s0 * npix, x, y, size, rot_cs[2 * j],
                                            rot_cs[2 * j + 1], b);
                    }
                }
                const long long r0 = s0 * num_rot + j0 - row_begin;
                if (j0 + 3 < num_rot && (r0 & 3) == 0 && r0 >= 0 && r0 + 3 < n_rows) {
                    reinterpret_cast<float4 *>(out)[((r0 >> 2) * n_parts + h) * part_w + cl] =
                        make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
                    for (int q = 0; q < 4; ++q) amax = fmaxf(amax, fabsf(v[q]));
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const long long r = r0 + q;
                        if (j0 + q >= num_rot || r < 0 || r >= n_rows) continue;
                        out[(((r >> 2) * n_parts + h) * part_w + cl) * 4 + (r & 3)] = v[q];
                        amax = fmaxf(amax, fabsf(v[q]));
                    }
                }
            }
        }
    }
    if (abs_max) {
        amax = __int_as_float(warp_max_int(__float_as_int(amax)));
        if ((threadIdx.x & 31) == 0)
            atomicMax(reinterpret_cast<int *>(abs_max), __float_as_int(amax));
    }
}

__global__ void __launch_bounds__(256)
k_rot_log_sets(const double2 *__restrict__ hp, int num_rot,
               const double *__restrict__ rot_cs, int size, const double *__restrict__ bg,
               const int *__restrict__ sel_pix, int n_sel, int n_parts, int part_w,
               long long row_begin, long long row_end, long long s_lo, float *__restrict__ out,
               float *__restrict__ abs_max) {
    const int n_jb = (num_rot + 3) / 4;
    const int j0 = (int)(blockIdx.x % (unsigned)n_jb) * 4;
    const long long s_first = s_lo + (long long)(blockIdx.x / (unsigned)n_jb) * RL_STATES;
    const long long npix = (long long)size * size;
    const long long n_rows = row_end - row_begin;
    const int cen = size / 2;
    const float inv_size = 1.f / (float)size;
    // this CTA's states with a row s0 * num_rot + j0 + q in [row_begin, row_end)
    long long sb = s_first, se = s_first + RL_STATES;
    while (sb < se && sb * num_rot + min(j0 + 3, num_rot - 1) < row_begin) ++sb;
    while (se > sb && (se - 1) * num_rot + j0 >= row_end) --se;
    double ac[4], as[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = min(j0 + q, num_rot - 1);
        ac[q] = rot_cs[2 * j];
        as[q] = rot_cs[2 * j + 1];
    }
    const int n_cols = n_parts * part_w;
    float amax = 0.f;
    if (sb < se) {
        for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
            const int h = c / part_w, cl = c - h * part_w;
            bool in[4] = {false, false, false, false};
            int base[4] = {0, 0, 0, 0};
            double fx[4] = {0., 0., 0., 0.}, fy[4] = {0., 0., 0., 0.};
            double b = 0.;
            if (c < n_sel) {
                const int p = sel_pix[c];
                int x, y;
                pixel_xy(p, size, inv_size, x, y);
                const double xc = (double)(x - cen), yc = (double)(y - cen);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double tx = xadd(xsub(xmul(xc, ac[q]), xmul(yc, as[q])), (double)cen);
                    const double ty = xadd(xadd(xmul(xc, as[q]), xmul(yc, ac[q])), (double)cen);
                    const double fxl = floor(tx), fyl = floor(ty);
                    in[q] = !(fxl < 0. || fxl > size - 2 || fyl < 0. || fyl > size - 2);
                    if (in[q]) {
                        base[q] = (int)fxl * size + (int)fyl;
                        fx[q] = tx - fxl;
                        fy[q] = ty - fyl;
                    }
                }
                b = bg[p];
            }
            for (long long s0 = sb; s0 < se; ++s0) {
                float v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    double val = 0.;
                    if (c < n_sel) {
                        if (in[q]) {
                            const double2 a = hp[s0 * npix + base[q]];
                            const double2 b2 = hp[s0 * npix + base[q] + size];
                            const double cx = 1. - fx[q], cy = 1. - fy[q];
                            double t = xmul(xmul(a.x, cx), cy);
                            t = xadd(t, xmul(xmul(b2.x, fx[q]), cy));
                            t = xadd(t, xmul(xmul(a.y, cx), fy[q]));
                            t = xadd(t, xmul(xmul(b2.y, fx[q]), fy[q]));
                            t = xadd(t, b);
                            val = t < 1.e-20 ? -1000. : log(t);
                        } else {
                            val = -1000.;
                        }
                    }
                    v[q] = (float)val;
                }
                const long long r0 = s0 * num_rot + j0 - row_begin;
                if (j0 + 3 < num_rot && (r0 & 3) == 0 && r0 >= 0 && r0 + 3 < n_rows) {
                    reinterpret_cast<float4 *>(out)[((r0 >> 2) * n_parts + h) * part_w + cl] =
                        make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
                    for (int q = 0; q < 4; ++q) amax = fmaxf(amax, fabsf(v[q]));
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const long long r = r0 + q;
                        if (j0 + q >= num_rot || r < 0 || r >= n_rows) continue;
                        out[(((r >> 2) * n_parts + h) * part_w + cl) * 4 + (r & 3)] = v[q];
                        amax = fmaxf(amax, fabsf(v[q]));
                    }
                }
            }
        }
    }
    if (abs_max) {
        amax = __int_as_float(warp_max_int(__float_as_int(amax)));
        if ((threadIdx.x & 31) == 0)
            atomicMax(reinterpret_cast<int *>(abs_max), __float_as_int(amax));
    }
}

}  // namespace

extern "C" int rspi_holo_slices(const double *model, const double *shiftx, const double *shifty,
                                const double *sphere_dia, long long n_states0, long long size,
                                const double *bg, const int *sel_pix, long long n_sel,
                                double *holo, double *msum, cudaStream_t stream) {
    if (n_states0 <= 0 || size <= 1 || n_sel < 0 || !model || !holo || !msum || !bg)
        return RSPI_ERR_ARG;
    if (n_states0 > 0x7fffffffLL) return RSPI_ERR_ARG;
    k_holo<<<(unsigned)n_states0, HOLO_THREADS, 0, stream>>>(
        (const double2 *)model, shiftx, shifty, sphere_dia, size, bg, sel_pix, n_sel, holo, msum);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_vscale_init(const double *msum, long long n_states0, const double *powder,
                                const int *sel_pix, long long n_sel, double *vscale,
                                double *init, cudaStream_t stream) {
    if (n_states0 <= 0 || n_sel < 0 || !msum || !powder || !vscale || !init) return RSPI_ERR_ARG;
    k_vscale_init<<<1, 1024, 0, stream>>>(msum, n_states0, powder, sel_pix, n_sel, vscale, init);
    RSPI_RETURN_LAUNCH();
}

template <bool PAIRS>
static int rot_log_launch(const double *holo, const double2 *hp, long long n_states0,
                          long long num_rot, const double *rot_cs, long long size,
                          const double *bg, const int *sel_pix, long long n_sel, long long p_pad,
                          long long row_begin, long long row_end, void *lslices, int out_dtype,
                          float *abs_max, cudaStream_t stream) {
    if (n_states0 <= 0 || num_rot <= 0 || size <= 1 || size > 46340 || p_pad < n_sel ||
        p_pad % 32 || row_begin < 0 || row_end > n_states0 * num_rot || row_end < row_begin ||
        !(PAIRS ? (const void *)hp : (const void *)holo) || !rot_cs || !bg || !lslices)
        return RSPI_ERR_ARG;
    if (PAIRS && (reinterpret_cast<uintptr_t>(hp) & 15) != 0) return RSPI_ERR_ARG;
    const long long n_rows = row_end - row_begin;
    if (n_rows == 0) return RSPI_OK;
    // rotation-major CTAs: one rotation, RL_STATES consecutive states
    const long long s_lo = row_begin / num_rot, s_hi = (row_end - 1) / num_rot;
    const long long n_groups = (s_hi - s_lo) / RL_STATES + 1;
    if (n_groups * num_rot > 0x7fffffffLL || p_pad > 0x7fffffffLL || n_sel > p_pad)
        return RSPI_ERR_ARG;
    const unsigned blocks = (unsigned)(n_groups * num_rot);
    if (out_dtype == 0)
        k_rot_log_js<float, PAIRS><<<blocks, 256, 0, stream>>>(
            holo, hp, (int)num_rot, rot_cs, (int)size, bg, sel_pix, (int)n_sel, (int)p_pad,
            row_begin, row_end, s_lo, (int)n_groups, (float *)lslices, abs_max);
    else if (out_dtype == 2)
        k_rot_log_js<__half, PAIRS><<<blocks, 256, 0, stream>>>(
            holo, hp, (int)num_rot, rot_cs, (int)size, bg, sel_pix, (int)n_sel, (int)p_pad,
            row_begin, row_end, s_lo, (int)n_groups, (__half *)lslices, abs_max);
    else if (out_dtype == 1)
        k_rot_log_js<double, PAIRS><<<blocks, 256, 0, stream>>>(
            holo, hp, (int)num_rot, rot_cs, (int)size, bg, sel_pix, (int)n_sel, (int)p_pad,
            row_begin, row_end, s_lo, (int)n_groups, (double *)lslices, abs_max);
    else
        return RSPI_ERR_ARG;
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rot_log_slices(const double *holo, long long n_states0, long long num_rot,
                                   const double *rot_cs, long long size, const double *bg,
                                   const int *sel_pix, long long n_sel, long long p_pad,
                                   long long row_begin, long long row_end, void *lslices,
                                   int out_dtype, float *abs_max, cudaStream_t stream) {
    return rot_log_launch<false>(holo, nullptr, n_states0, num_rot, rot_cs, size, bg, sel_pix,
                                 n_sel, p_pad, row_begin, row_end, lslices, out_dtype, abs_max,
                                 stream);
}

extern "C" int rspi_holo_pairs(const double *holo, long long n_states0, long long size,
                               double *holo_pairs, cudaStream_t stream) {
    if (!holo || !holo_pairs || n_states0 <= 0 || size <= 1 || size > 46340 ||
        (reinterpret_cast<uintptr_t>(holo_pairs) & 15) != 0)
        return RSPI_ERR_ARG;
    const long long total = n_states0 * size * size;
    k_holo_pairs<<<rspi_blocks(total, 256), 256, 0, stream>>>(
        holo, total, reinterpret_cast<double2 *>(holo_pairs));
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rot_log_slices_pairs(const double *holo_pairs, long long n_states0,
                                         long long num_rot, const double *rot_cs, long long size,
                                         const double *bg, const int *sel_pix, long long n_sel,
                                         long long p_pad, long long row_begin, long long row_end,
                                         void *lslices, int out_dtype, float *abs_max,
                                         cudaStream_t stream) {
    return rot_log_launch<true>(nullptr, reinterpret_cast<const double2 *>(holo_pairs),
                                n_states0, num_rot, rot_cs, size, bg, sel_pix, n_sel, p_pad,
                                row_begin, row_end, lslices, out_dtype, abs_max, stream);
}

extern "C" int rspi_sphere_ramp(long long size, double sx, double sy, double dia, double *sphere,
                                double *ramp, cudaStream_t stream) {
    if (size <= 1 || size > 46340 || (!sphere && !ramp)) return RSPI_ERR_ARG;
    k_sphere_ramp<<<rspi_blocks(size * size, 256), 256, 0, stream>>>(
        (int)size, sx, sy, dia, sphere, (double2 *)ramp);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_holo_quads32(const double *holo, long long n_states0, long long size,
                                 float *holo_quads32, cudaStream_t stream) {
    if (!holo || !holo_quads32 || n_states0 <= 0 || size <= 1 || size > 46340 ||
        (reinterpret_cast<uintptr_t>(holo_quads32) & 15) != 0)
        return RSPI_ERR_ARG;
    const long long total = n_states0 * size * size;
    k_holo_quads32<<<rspi_blocks(total, 256), 256, 0, stream>>>(
        holo, total, (int)size, reinterpret_cast<float4 *>(holo_quads32));
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rot_log_slices_sets(const double *holo_pairs, const float *holo_quads32,
                                        long long n_states0, long long num_rot,
                                        const double *rot_cs, long long size, const double *bg,
                                        const int *sel_pix, long long n_sel, int n_parts,
                                        int part_w, long long row_begin, long long row_end,
                                        float *out, float *abs_max, cudaStream_t stream) {
    if (!holo_pairs || !rot_cs || !bg || !out || n_states0 <= 0 || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || size <= 1 || size > 46340 || n_sel < 0 || n_parts < 1 ||
        part_w < 1 || (long long)n_parts * part_w < n_sel ||
        (long long)n_parts * part_w > 0x7fffffffLL || row_begin < 0 || row_end < row_begin ||
        row_end > n_states0 * num_rot || (n_sel > 0 && !sel_pix) ||
        (reinterpret_cast<uintptr_t>(holo_pairs) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(holo_quads32) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(out) & 15) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const long long s_lo = row_begin / num_rot, s_hi = (row_end - 1) / num_rot;
    const long long n_groups = (s_hi - s_lo) / RL_STATES + 1;
    const long long n_jb = (num_rot + 3) / 4;
    if (n_groups * n_jb > 0x7fffffffLL) return RSPI_ERR_ARG;
    const double2 *hp = reinterpret_cast<const double2 *>(holo_pairs);
    const float4 *hq = reinterpret_cast<const float4 *>(holo_quads32);
    if (hq)
        k_rot_log_sets32<<<(unsigned)(n_groups * n_jb), 1024, 0, stream>>>(
            hp, hq, (int)num_rot, rot_cs, (int)size, bg, sel_pix, (int)n_sel, n_parts, part_w,
            row_begin, row_end, s_lo, out, abs_max);
    else
        k_rot_log_sets<<<(unsigned)(n_groups * n_jb), 256, 0, stream>>>(
            hp, (int)num_rot, rot_cs, (int)size, bg, sel_pix, (int)n_sel, n_parts, part_w,
            row_begin, row_end, s_lo, out, abs_max);
    RSPI_RETURN_LAUNCH();
}
