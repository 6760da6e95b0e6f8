// MaxLP M-step (rows a11-a14): per-pixel complex pattern search.
//
// The reference (maxLP.py:154-197) evaluates, for every model pixel and each
// of 1089 candidates f_c, mean over ALL frames of k_d log(rho |f_c + r_d|^2)
// minus mean of rho |f_c + r_d|^2, materialising frames x candidates arrays
// (~20 CuPy launches per pattern iteration).  Two exact rewrites make it a
// per-pixel register computation here:
//  * r_d depends on frame d only through its reference state (shift,
//    diameter), so frames sharing a state share the log term:
//      sum_d k_d log(rho w_d) = sum_s K_t[s] log(rho |f_c + r_s|^2),
//    with K_t[s] the photons that pixel t receives from frames in state s
//    (built once per M-step by scattering each photon to the model pixels
//    whose rotated index lands on it);
//  * the frame mean of |f_c + r_d|^2 is |f_c + rbar|^2 + var(r), with
//    rbar = mean_d r_d and var(r) = mean_d |r_d - rbar|^2 per pixel.
// All arithmetic is FP64, so candidate values agree with the FP64
// restatement to rounding and the search takes the same path.
#include "rspi_common.cuh"

namespace {

constexpr double PI = 3.14159265358979311599796346854;  // the double nearest pi
constexpr int NCAND = 1089;                               // 33 x 33 (maxLP.py:45-48)
constexpr int CENTRE = NCAND / 2;                         // maxLP.py:176
constexpr int PT_THREADS = 384;
constexpr int PT_CPT = 3;                                 // 384 * 3 >= 1089
constexpr int POP_CAP = 1024;                             // populated states in shared memory

__global__ void k_frame_params(const int *__restrict__ rmax, long long n, long long num_rot,
                               long long n_ref, int *__restrict__ fstate, int *__restrict__ frot,
                               int *__restrict__ nstate, int *err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        const long long r = rmax[d];
        if (r < 0 || r >= n_ref * num_rot) {
            rspi_flag(err, RSPI_ERR_INDEX);
            fstate[d] = -1;
            frot[d] = 0;
            continue;
        }
        const int s = (int)(r / num_rot);
        fstate[d] = s;
        frot[d] = (int)(r - (long long)s * num_rot);
        atomicAdd(&nstate[s], 1);
    }
}

// Add `cnt` photons at detector (ux, uy) to every phaser pixel that maps
// onto exactly (ux, uy).  Such pixels lie within 1/sqrt(2) px of the inverse
// image, so the 3x3 neighbourhood of its rounding holds them all.
__device__ __forceinline__ void scatter_photon(int ux, int uy, int cnt, double c, double s,
                                               int size, const int *__restrict__ mask_idx,
                                               long long n_ref, int st, int *__restrict__ hist) {
    const double c0 = (double)(size / 2);
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
            if (ox == ux && oy == uy) atomicAdd(&hist[(long long)m * n_ref + st], cnt);
        }
}

__global__ void __launch_bounds__(256)
k_histogram(const int *__restrict__ ones, const int *__restrict__ multi,
            const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
            const int *__restrict__ place_ones, const int *__restrict__ place_multi,
            const int *__restrict__ count_multi, long long n, const int *__restrict__ fstate,
            const int *__restrict__ frot, const double *__restrict__ rot_cs, int size,
            const int *__restrict__ mask_idx, long long n_ref, int *__restrict__ hist, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long npix = (long long)size * size;
    for (long long d = warp; d < n; d += nwarp) {
        const int st = fstate[d];
        if (st < 0) continue;
        const int j = frot[d];
        const double c = rot_cs[2 * j], s = rot_cs[2 * j + 1];
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
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
            scatter_photon(ux, uy, cnt, c, s, size, mask_idx, n_ref, st, hist);
            // column x*size + size of row x aliases pixel (x+1, 0): even sizes only
            if (uy == 0 && ux >= 1 && (size % 2) == 0)
                scatter_photon(ux - 1, size, cnt, c, s, size, mask_idx, n_ref, st, hist);
        }
    }
}

// The same histogram from a table built once per rotation table: for each
// rotation j and detector pixel p, the phaser rows whose pixel's forward
// map lands on p (the 3 x 3 search of scatter_photon finds exactly these,
// since such pixels lie within 1/sqrt(2) px of p's inverse image).  A pixel
// whose map lands on column `size` of row x (even sizes) is listed under
// pixel (x + 1, 0), as scatter_photon aliases it.  Per photon the histogram
// then reads its table range instead of nine forward maps.
__device__ __forceinline__ long long map_key(int tx, int ty, double c, double s, int size) {
    int ox, oy;
    forward_pixel(tx, ty, c, s, size, ox, oy);
    if (ox >= 0 && ox < size && oy >= 0 && oy < size) return (long long)ox * size + oy;
    if ((size % 2) == 0 && oy == size && ox >= 0 && ox + 1 < size)
        return (long long)(ox + 1) * size;
    return -1;
}

__global__ void k_pixel_map_count(const double *__restrict__ rot_cs, long long num_rot, int size,
                                  const int *__restrict__ mask_idx, int *__restrict__ cnt) {
    const long long npix = (long long)size * size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < num_rot * npix;
         i += stride) {
        const long long j = i / npix, t = i - j * npix;
        if (mask_idx[t] < 0) continue;
        const long long key = map_key((int)(t / size), (int)(t % size), rot_cs[2 * j],
                                      rot_cs[2 * j + 1], size);
        if (key >= 0) atomicAdd(&cnt[j * npix + key], 1);
    }
}

__global__ void k_pixel_map_fill(const double *__restrict__ rot_cs, long long num_rot, int size,
                                 const int *__restrict__ mask_idx,
                                 const long long *__restrict__ off, int *__restrict__ cursor,
                                 int *__restrict__ rows) {
    const long long npix = (long long)size * size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < num_rot * npix;
         i += stride) {
        const long long j = i / npix, t = i - j * npix;
        const int m = mask_idx[t];
        if (m < 0) continue;
        const long long key = map_key((int)(t / size), (int)(t % size), rot_cs[2 * j],
                                      rot_cs[2 * j + 1], size);
        if (key < 0) continue;
        const long long k = j * npix + key;
        rows[off[k] + atomicAdd(&cursor[k], 1)] = m;   // order within a pixel: any (integer sums)
    }
}

__global__ void __launch_bounds__(256)
k_histogram_map(const int *__restrict__ ones, const int *__restrict__ multi,
                const long long *__restrict__ ones_accum, const long long *__restrict__ multi_accum,
                const int *__restrict__ place_ones, const int *__restrict__ place_multi,
                const int *__restrict__ count_multi, long long n, const int *__restrict__ fstate,
                const int *__restrict__ frot, long long num_rot, int size,
                const long long *__restrict__ map_off, const int *__restrict__ map_rows,
                long long n_ref, int *__restrict__ hist, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long npix = (long long)size * size;
    for (long long d = warp; d < n; d += nwarp) {
        const int st = fstate[d];
        if (st < 0) continue;
        const int j = frot[d];
        if (j < 0 || j >= num_rot) {
            rspi_flag(err, RSPI_ERR_INDEX);
            continue;
        }
        const long long *off = map_off + (long long)j * npix;
        const int n_o = ones[d], n_m = multi[d];
        const long long oa = ones_accum[d], ma = multi_accum[d];
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
            for (long long e = off[p]; e < off[p + 1]; ++e)
                atomicAdd(&hist[(long long)map_rows[e] * n_ref + st], cnt);
        }
    }
}

// Reference-sphere amplitude at pixel (qx, qy, qrad) for state (sx, sy, dia),
// maxLP.py:238-243: ff(pi qrad dia) exp(2 pi i (qx sx + qy sy)).
__device__ __forceinline__ double2 fref_value(double qx, double qy, double qrad, double sx,
                                              double sy, double dia) {
    const double sval = xmul(xmul(PI, qrad), dia);
    const double ff = xsub(sin(sval), xmul(sval, cos(sval))) / pow(sval, 3.);
    const double th = xmul(2. * PI, xadd(xmul(qx, sx), xmul(qy, sy)));
    return make_double2(ff * cos(th), ff * sin(th));
}

struct PixelConsts {
    double qx, qy, qrad;
    double ar, ai;   // rbar = mean_d r_d
    double var;      // mean_d |r_d - rbar|^2
    double ksum;     // sum_d k_d
};

__device__ __forceinline__ void block_argmax(double &v, int &idx, double *sv, int *si) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(RSPI_FULL_MASK, v, o);
        const int oi = __shfl_xor_sync(RSPI_FULL_MASK, idx, o);
        if (argmax_better(ov, oi, v, idx)) {
            v = ov;
            idx = oi;
        }
    }
    __syncthreads();
    if (lane == 0) {
        sv[wid] = v;
        si[wid] = idx;
    }
    __syncthreads();
    if (wid == 0) {
        double bv = lane < nw ? sv[lane] : 0.;
        int bi = lane < nw ? si[lane] : 0x7fffffff;
        if (lane >= nw) bv = -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(RSPI_FULL_MASK, bv, o);
            const int oi = __shfl_xor_sync(RSPI_FULL_MASK, bi, o);
            if (argmax_better(ov, oi, bv, bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sv[0] = bv;
            si[0] = bi;
        }
    }
    __syncthreads();
    v = sv[0];
    idx = si[0];
    __syncthreads();
}

// Ordered compaction of the populated reference states of one pixel, from
// state `s_begin` on, into shared memory (at most POP_CAP).  Returns the state
// where the next chunk starts (n_ref when done); *count gets the number stored.
__device__ int load_populated(int s_begin, const int *__restrict__ hrow, long long n_ref,
                              const double *__restrict__ ref_params, const PixelConsts &pc,
                              double *fr_re, double *fr_im, double *fk, int *count, int *wsum) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    int filled = 0;
    int s0 = s_begin;
    while (s0 < n_ref) {
        const int s = s0 + threadIdx.x;
        const int h = s < n_ref ? hrow[s] : 0;
        const unsigned bal = __ballot_sync(RSPI_FULL_MASK, h > 0);
        __syncthreads();
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        int before = 0, round = 0;
        for (int w = 0; w < nw; ++w) {
            if (w < wid) before += wsum[w];
            round += wsum[w];
        }
        if (filled + round > POP_CAP) break;  // this round starts the next chunk
        if (h > 0) {
            const int pos = filled + before + __popc(bal & ((1u << lane) - 1u));
            const double2 r = fref_value(pc.qx, pc.qy, pc.qrad, ref_params[3 * s],
                                         ref_params[3 * s + 1], ref_params[3 * s + 2]);
            fr_re[pos] = r.x;
            fr_im[pos] = r.y;
            fk[pos] = (double)h;
        }
        filled += round;
        s0 += blockDim.x;
    }
    __syncthreads();
    *count = filled;
    return s0 < n_ref ? s0 : (int)n_ref;
}

// One candidate of the 33 x 33 pattern around f (maxLP.py:45-48,168-170):
// its value, the frame mean of |f_c + r_d|^2 (|f_c + rbar|^2 + var) and its
// rescale (the ring pass: mean photons / that mean, maxLP.py:216-228;
// the main pass: the ring's mean rescale).  Explicit roundings, so the plain
// and the screened search compute the same bits.
struct Cand {
    double fr, fi, mw, rho;
};

__device__ __forceinline__ Cand cand_at(int c, double2 f, double step, const PixelConsts &pc,
                                        bool ring, double kmean, double rescale) {
    const double px = -8. + 0.5 * (c / 33), py = -8. + 0.5 * (c % 33);
    Cand o;
    o.fr = xadd(f.x, xmul(px, step));
    o.fi = xadd(f.y, xmul(py, step));
    const double er = xadd(o.fr, pc.ar), ei = xadd(o.fi, pc.ai);
    o.mw = fma(er, er, fma(ei, ei, pc.var));
    o.rho = ring ? kmean / o.mw : rescale;
    return o;
}

// acc + k log(rho |f_c + r|^2): one populated state's term (maxLP.py:181-197).
__device__ __forceinline__ double term64(double acc, double kk, const Cand &c, double rr,
                                         double ri) {
    const double re = xadd(c.fr, rr), im = xadd(c.fi, ri);
    return fma(kk, log(xmul(c.rho, fma(re, re, xmul(im, im)))), acc);
}

// The candidate's value: frame mean of the log term minus the mean rescaled
// intensity.
__device__ __forceinline__ double cand_q(double acc, double dn, const Cand &c) {
    return xsub(acc / dn, xmul(c.rho, c.mw));
}

// A candidate's log term is summed as NPART partial sums, the p-th over the
// populated states j = p, p + NPART, ... of a chunk in order, combined as
// (s0 + s1) + (s2 + s3): the plain search keeps the four in registers, the
// screened search's finalists give each to its own thread.
__device__ __forceinline__ double combine4(double s0, double s1, double s2, double s3) {
    return xadd(xadd(s0, s1), xadd(s2, s3));
}

// Adds one chunk of npop populated states to a candidate's NPART partial
// sums (state j of the chunk to sum j mod NPART).
__device__ __forceinline__ void sum_partials(double (&acc)[4], const Cand &ck, int npop,
                                             const double *fr_re, const double *fr_im,
                                             const double *fk) {
    double a0 = acc[0], a1 = acc[1], a2 = acc[2], a3 = acc[3];
    int j = 0;
    for (; j + 4 <= npop; j += 4) {
        a0 = term64(a0, fk[j], ck, fr_re[j], fr_im[j]);
        a1 = term64(a1, fk[j + 1], ck, fr_re[j + 1], fr_im[j + 1]);
        a2 = term64(a2, fk[j + 2], ck, fr_re[j + 2], fr_im[j + 2]);
        a3 = term64(a3, fk[j + 3], ck, fr_re[j + 3], fr_im[j + 3]);
    }
    if (j < npop) a0 = term64(a0, fk[j], ck, fr_re[j], fr_im[j]);
    if (j + 1 < npop) a1 = term64(a1, fk[j + 1], ck, fr_re[j + 1], fr_im[j + 1]);
    if (j + 2 < npop) a2 = term64(a2, fk[j + 2], ck, fr_re[j + 2], fr_im[j + 2]);
    acc[0] = a0;
    acc[1] = a1;
    acc[2] = a2;
    acc[3] = a3;
}

__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Error of lg2.approx.f32 for x in [2^-100, 2^100]:
//   |lg2(x) - log2(x)| <= LG2_EA + LG2_ER |lg2(x)|,
// checked over every float of that range by rspi_log2_error_max.
constexpr double LG2_EA = 0x1p-21;
constexpr double LG2_ER = 0x1p-22;
constexpr double U32 = 0x1p-24;                    // FP32 unit roundoff
constexpr double LN2 = 0x1.62e42fefa39efp-1;       // the double nearest ln 2
constexpr int PT_CHUNK = 32;                       // FP32 terms per FP64 add
constexpr double G_CHUNK = 32.01 * U32;            // gamma_32 (+ the FP64 adds)
constexpr int NPART = 4;                           // partial sums per candidate
static_assert(NPART == 4, "combine4 and sum_partials take four partial sums");
constexpr int FIN_SPLIT = PT_THREADS / NPART;      // up to here: NPART threads each
constexpr int FIN_CAP = NCAND;                     // beyond: a thread per finalist,
                                                   // NPART sums, up to PT_CPT each

__device__ __forceinline__ double block_max_d(double v, double *scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(RSPI_FULL_MASK, v, o));
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double m = -INFINITY;
    for (int w = 0; w < nw; ++w) m = fmax(m, scratch[w]);
    __syncthreads();
    return m;
}

// Exclusive prefix of v in thread order, and the block total in *total.
__device__ __forceinline__ int block_scan(int v, int *wsum, int *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(RSPI_FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    int before = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
        if (w < wid) before += wsum[w];
        tot += wsum[w];
    }
    __syncthreads();
    *total = tot;
    return before + x - v;
}

// One FP32 screening term for a candidate held as hi + lo parts (xh, xl:
// (real, imaginary)) against a populated state r = (re hi, im hi, re lo,
// im lo), everything scaled by the pixel's power of two.  The real and
// imaginary parts go through the packed FP32x2 adds (each lane rounded on
// its own), and ab = (sum k l, sum k |l|) through one packed FMA.
__device__ __forceinline__ void screen_term(float2 xh, float2 xl, const float4 r, float kj,
                                            float &gmin, float2 &ab) {
    const float2 z = __fadd2_rn(__fadd2_rn(xh, make_float2(r.x, r.y)),
                                __fadd2_rn(xl, make_float2(r.z, r.w)));
    const float g = fmaf(z.x, z.x, __fmul_rn(z.y, z.y));
    gmin = fminf(gmin, g);
    const float l = lg2_approx(g);
    ab = __ffma2_rn(make_float2(kj, kj), make_float2(l, fabsf(l)), ab);
}

// Per-pixel pattern search (maxLP.py:154-179, 304-340): one CTA per phaser
// pixel (x mode), every thread PT_CPT candidates, the populated reference
// states of the pixel in shared memory.
//
// SCREEN: each iteration first evaluates every candidate in FP32 (hi + lo
// differences, lg2.approx, chunked sums) with a rigorous bound E_c on its
// distance from the FP64 value; only the finalists, the candidates whose
// upper end q32 + E reaches the best lower end max(q32 - E), are evaluated
// in FP64 with the plain search's sums (four partial sums each, on four
// threads or one).  The FP64 argmax is always a finalist and every other
// candidate's FP64 value is strictly below it, so the chosen candidate is
// the plain search's.  A candidate without a finite bound is a finalist.  A
// pixel runs the plain FP64 iterations when it has more than one chunk of
// populated states, counts >= 2^24, or is a ring pixel without photons.
//
// Bound, per term (u = 2^-24; A = |f_c|_inf + max_s |r_s|_inf, scaled):
//   re, im from hi + lo parts: error <= 2u |re| + 6 u^2 A, so while
//   |f_c + r|^2 >= max(2^-24 A^2, 2^-100) (checked through the minimum g):
//   |ln g32 - ln g| <= 6.5 u, i.e. 9.5 u in log2;
//   lg2: LG2_EA + LG2_ER |l|; chunk sums: gamma_32 sum k |l|.
//   E_c = ln2 (K (LG2_EA + 9.5u) + (LG2_ER + g32)(1 + g32) sum k|l|) / n
//         + 2^-40 (FP64 rounding of both evaluations).
template <bool SCREEN>
__global__ void __launch_bounds__(PT_THREADS, 2)
k_pattern(double2 *__restrict__ fconv, const int *__restrict__ pixels,
          const int *__restrict__ hist_row, long long n_pix, const int *__restrict__ hist,
          long long n_ref, const int *__restrict__ nstate, long long n_modes,
          const double *__restrict__ ref_params, int size, int ring,
          const double *__restrict__ rescale_ptr, int num_iter, double *__restrict__ rescale_out,
          unsigned long long *__restrict__ stats) {
    __shared__ double fr_re[POP_CAP], fr_im[POP_CAP], fk[POP_CAP];
    __shared__ float4 r32[SCREEN ? POP_CAP : 1];
    __shared__ float k32[SCREEN ? POP_CAP : 1];
    __shared__ short fin[SCREEN ? FIN_CAP : 1];
    __shared__ double scratch[32];
    __shared__ int iscratch[32];
    __shared__ int wsum[32];

    // blockIdx.y = mode: its model, its histogram columns, its frames
    const long long mode = blockIdx.y;
    const long long ip = blockIdx.x;
    const int t = pixels[ip];
    const int *hrow = hist + (long long)hist_row[ip] * n_ref * n_modes + mode * n_ref;
    nstate += mode * n_ref;
    fconv += mode * (long long)size * size;
    // frames of this mode (all frames for one mode): an exact integer sum
    double cnt = 0.;
    for (long long s = threadIdx.x; s < n_ref; s += blockDim.x) cnt += (double)nstate[s];
    const double dn = block_sum(cnt, scratch);
    if (dn == 0.) {  // no frame chose this mode: its model stays as it is
        if (threadIdx.x == 0 && rescale_out) rescale_out[mode * n_pix + ip] = NAN;
        return;
    }

    PixelConsts pc;
    {
        const double ds = (double)size, c0 = (double)(size / 2);
        const int tx = t / size, ty = t - (t / size) * size;
        pc.qx = ((double)tx - c0) / ds;
        pc.qy = ((double)ty - c0) / ds;
        pc.qrad = sqrt(xadd(xmul(pc.qx, pc.qx), xmul(pc.qy, pc.qy)));
        if (pc.qrad == 0.) pc.qrad = 1.e-6;  // maxLP.py:85
    }
    // rbar, K total
    double ar = 0., ai = 0., ks = 0.;
    for (long long s = threadIdx.x; s < n_ref; s += blockDim.x) {
        const int ns = nstate[s];
        ks += (double)hrow[s];
        if (ns > 0) {
            const double2 r = fref_value(pc.qx, pc.qy, pc.qrad, ref_params[3 * s],
                                         ref_params[3 * s + 1], ref_params[3 * s + 2]);
            ar = fma((double)ns, r.x, ar);
            ai = fma((double)ns, r.y, ai);
        }
    }
    pc.ar = block_sum(ar, scratch) / dn;
    pc.ai = block_sum(ai, scratch) / dn;
    pc.ksum = block_sum(ks, scratch);
    double vv = 0.;
    for (long long s = threadIdx.x; s < n_ref; s += blockDim.x) {
        const int ns = nstate[s];
        if (ns > 0) {
            const double2 r = fref_value(pc.qx, pc.qy, pc.qrad, ref_params[3 * s],
                                         ref_params[3 * s + 1], ref_params[3 * s + 2]);
            const double er = xsub(r.x, pc.ar), ei = xsub(r.y, pc.ai);
            vv = fma((double)ns, fma(er, er, xmul(ei, ei)), vv);
        }
    }
    pc.var = block_sum(vv, scratch) / dn;

    int npop = 0;
    const bool one_chunk = n_ref <= POP_CAP;
    if (one_chunk) load_populated(0, hrow, n_ref, ref_params, pc, fr_re, fr_im, fk, &npop, wsum);

    const double kmean = pc.ksum / dn;
    const double rescale = ring ? 0. : rescale_ptr[mode];
    // screen bound constants: the main pass's rho is the ring's mean rescale
    // for every candidate, so its log is taken once per pixel; the bound
    // multiplies by 1/dn (at most two ulps of q and e beyond the divisions,
    // far inside its 2^-40 term)
    const double inv_dn = 1. / dn;
    const double lr_main = ring ? 0. : log(rescale);
    double2 f = fconv[t];
    double step = hypot(f.x, f.y) / 4.;
    const double shrink = 33. / 5.;  // sqrt(1089) / 5, maxLP.py:177

    // FP32 copies of the populated states, scaled by 2^-sexp so that the
    // largest of |f|_inf and max |r|_inf lies in [1/2, 1)
    bool screen = false;
    int sexp = 0;
    double sc = 1., rinf_s = 0.;
    if (SCREEN && one_chunk && !(ring && pc.ksum == 0.)) {
        double rl = 0.;
        int bad = 0;
        for (int j = threadIdx.x; j < npop; j += blockDim.x) {
            rl = fmax(rl, fmax(fabs(fr_re[j]), fabs(fr_im[j])));
            bad |= !(fk[j] < 16777216.);
        }
        bad = __syncthreads_or(bad);
        rl = block_max_d(rl, scratch);
        const double top = fmax(rl, fmax(fabs(f.x), fabs(f.y)));
        if (!bad && top > 0x1p-1000 && top < 0x1p1000) {
            frexp(top, &sexp);
            sc = ldexp(1., -sexp);
            rinf_s = rl * sc;
            for (int j = threadIdx.x; j < npop; j += blockDim.x) {
                const double xr = fr_re[j] * sc, xi = fr_im[j] * sc;
                const float hr = (float)xr, hi = (float)xi;
                r32[j] = make_float4(hr, hi, (float)(xr - (double)hr), (float)(xi - (double)hi));
                k32[j] = (float)fk[j];
            }
            __syncthreads();
            screen = true;
        }
    }

    for (int it = 0; it < num_iter; ++it) {
        Cand cd[PT_CPT];
#pragma unroll
        for (int k = 0; k < PT_CPT; ++k) {
            const int c = threadIdx.x + k * PT_THREADS;
            cd[k] = cand_at(c < NCAND ? c : 0, f, step, pc, ring, kmean, rescale);
        }
        double best = -INFINITY;
        int bidx = 0x7fffffff;
        bool searched = false;
        if (SCREEN && screen) {
            float2 xh[PT_CPT], xl[PT_CPT];
            float gmin[PT_CPT];
            double a64[PT_CPT], b64[PT_CPT];
#pragma unroll
            for (int k = 0; k < PT_CPT; ++k) {
                const double xs = cd[k].fr * sc, ys = cd[k].fi * sc;
                xh[k] = make_float2((float)xs, (float)ys);
                xl[k] = make_float2((float)(xs - (double)xh[k].x), (float)(ys - (double)xh[k].y));
                gmin[k] = INFINITY;
                a64[k] = 0.;
                b64[k] = 0.;
            }
            int j = 0;
            for (; j + PT_CHUNK <= npop; j += PT_CHUNK) {
                float2 ab[PT_CPT];
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) ab[k] = make_float2(0.f, 0.f);
#pragma unroll 2
                for (int jj = 0; jj < PT_CHUNK; ++jj) {
                    const float4 r = r32[j + jj];
                    const float kj = k32[j + jj];
#pragma unroll
                    for (int k = 0; k < PT_CPT; ++k) screen_term(xh[k], xl[k], r, kj, gmin[k], ab[k]);
                }
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) {
                    a64[k] += (double)ab[k].x;
                    b64[k] += (double)ab[k].y;
                }
            }
            {
                float2 ab[PT_CPT];
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) ab[k] = make_float2(0.f, 0.f);
                for (; j < npop; ++j) {
                    const float4 r = r32[j];
                    const float kj = k32[j];
#pragma unroll
                    for (int k = 0; k < PT_CPT; ++k) screen_term(xh[k], xl[k], r, kj, gmin[k], ab[k]);
                }
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) {
                    a64[k] += (double)ab[k].x;
                    b64[k] += (double)ab[k].y;
                }
            }
            // each candidate's interval [lo, hi] around its FP64 value
            double lo[PT_CPT], up[PT_CPT];
            const double ksum = pc.ksum, e2 = 2. * (double)sexp;
#pragma unroll
            for (int k = 0; k < PT_CPT; ++k) {
                const int c = threadIdx.x + k * PT_THREADS;
                lo[k] = -INFINITY;
                up[k] = -INFINITY;
                if (c >= NCAND) continue;
                const double xs = cd[k].fr * sc, ys = cd[k].fi * sc;
                const double amax = fmax(fabs(xs), fabs(ys)) + rinf_s;
                const double thr = fmax(0x1p-24 * amax * amax, 0x1p-100);
                const double rho = cd[k].rho, mwv = cd[k].mw;
                bool safe = isfinite(a64[k]) && isfinite(b64[k]) && (double)gmin[k] >= thr &&
                            amax >= 0x1p-38 && amax <= 0x1p60 && rho > 0. && rho < INFINITY &&
                            isfinite(mwv);
                if (safe) {
                    const double lr = ring ? log(rho) : lr_main;
                    const double q = (ksum * lr + LN2 * (a64[k] + e2 * ksum)) * inv_dn - rho * mwv;
                    const double b2 = ksum * (LG2_EA + 9.5 * U32) +
                                      (LG2_ER + G_CHUNK) * (1. + G_CHUNK) * b64[k];
                    const double fm = 0x1p-40 * ((ksum * (fabs(lr) + LN2 * fabs(e2) + 1.) +
                                                  LN2 * 1.01 * b64[k]) * inv_dn +
                                                 fabs(rho * mwv));
                    const double e = 1.001 * LN2 * b2 * inv_dn + fm;
                    safe = isfinite(q) && isfinite(e);
                    lo[k] = q - e;
                    up[k] = q + e;
                }
                if (!safe) {
                    lo[k] = -INFINITY;
                    up[k] = INFINITY;
                }
            }
            double tl = -INFINITY;
#pragma unroll
            for (int k = 0; k < PT_CPT; ++k) tl = fmax(tl, lo[k]);
            tl = block_max_d(tl, scratch);
            int mine = 0;
#pragma unroll
            for (int k = 0; k < PT_CPT; ++k) mine += (threadIdx.x + k * PT_THREADS < NCAND) && up[k] >= tl;
            int nfin = 0;
            int pos = block_scan(mine, wsum, &nfin);
            // every candidate whose upper end reaches tl is a finalist (all
            // of them when no candidate has a finite bound: tl = -inf)
            {
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) {
                    const int c = threadIdx.x + k * PT_THREADS;
                    if (c < NCAND && up[k] >= tl) fin[pos++] = (short)c;
                }
                __syncthreads();
                if (nfin <= FIN_SPLIT) {
                    // NPART consecutive threads per finalist, thread p summing
                    // the states j = p mod NPART in order
                    const int fi = threadIdx.x / NPART, part = threadIdx.x % NPART;
                    double acc = 0.;
                    Cand cc;
                    if (fi < nfin) {
                        cc = cand_at(fin[fi], f, step, pc, ring, kmean, rescale);
                        for (int s = part; s < npop; s += NPART)
                            acc = term64(acc, fk[s], cc, fr_re[s], fr_im[s]);
                    }
                    const double v1 = __shfl_down_sync(RSPI_FULL_MASK, acc, 1);
                    const double v2 = __shfl_down_sync(RSPI_FULL_MASK, acc, 2);
                    const double v3 = __shfl_down_sync(RSPI_FULL_MASK, acc, 3);
                    if (fi < nfin && part == 0) {
                        best = cand_q(combine4(acc, v1, v2, v3), dn, cc);
                        bidx = fin[fi];
                    }
                } else {
                    // one thread per finalist, its NPART sums in registers
                    for (int i = threadIdx.x; i < nfin; i += PT_THREADS) {
                        const int c = fin[i];
                        const Cand cc = cand_at(c, f, step, pc, ring, kmean, rescale);
                        double a4[NPART] = {0., 0., 0., 0.};
                        sum_partials(a4, cc, npop, fr_re, fr_im, fk);
                        const double q = cand_q(combine4(a4[0], a4[1], a4[2], a4[3]), dn, cc);
                        if (argmax_better(q, c, best, bidx)) {
                            best = q;
                            bidx = c;
                        }
                    }
                }
                searched = true;
                if (stats && threadIdx.x == 0) {
                    atomicAdd(&stats[0], 1ull);
                    atomicAdd(&stats[2], (unsigned long long)nfin);
                }
            }
        }
        if (!searched) {
            // candidate by candidate (few live registers), each with its
            // NPART partial sums: four independent logs in flight
            double acc[PT_CPT][NPART];
            if (one_chunk) {
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k) {
                    double a4[NPART] = {0., 0., 0., 0.};
                    sum_partials(a4, cd[k], npop, fr_re, fr_im, fk);
                    acc[k][0] = combine4(a4[0], a4[1], a4[2], a4[3]);
                }
            } else {
                double part[PT_CPT][NPART];
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k)
#pragma unroll
                    for (int p = 0; p < NPART; ++p) part[k][p] = 0.;
                int s_next = 0;
                do {
                    s_next = load_populated(s_next, hrow, n_ref, ref_params, pc, fr_re, fr_im, fk,
                                            &npop, wsum);
#pragma unroll
                    for (int k = 0; k < PT_CPT; ++k)
                        sum_partials(part[k], cd[k], npop, fr_re, fr_im, fk);
                    __syncthreads();
                } while (s_next < n_ref);
#pragma unroll
                for (int k = 0; k < PT_CPT; ++k)
                    acc[k][0] = combine4(part[k][0], part[k][1], part[k][2], part[k][3]);
            }
#pragma unroll
            for (int k = 0; k < PT_CPT; ++k) {
                const int c = threadIdx.x + k * PT_THREADS;
                if (c >= NCAND) continue;
                double q = cand_q(acc[k][0], dn, cd[k]);
                if (ring && pc.ksum == 0.) q = NAN;  // 0 * log(0) in every frame
                if (argmax_better(q, c, best, bidx)) {
                    best = q;
                    bidx = c;
                }
            }
            if (SCREEN && stats && threadIdx.x == 0) atomicAdd(&stats[1], 1ull);
        }
        block_argmax(best, bidx, scratch, iscratch);
        const double px = -8. + 0.5 * (bidx / 33), py = -8. + 0.5 * (bidx % 33);
        const double2 fnew = make_double2(xadd(f.x, xmul(px, step)), xadd(f.y, xmul(py, step)));
        const double step_new = bidx == CENTRE ? step / shrink : step;
        if (step_new / hypot(fnew.x, fnew.y) < 1.e-3) break;  // keeps f (maxLP.py:162-165)
        f = fnew;
        step = step_new;
    }
    if (threadIdx.x == 0) {
        fconv[t] = f;
        if (rescale_out) {   // maxLP.py:328, with the candidates' explicit roundings
            const double er = xadd(f.x, pc.ar), ei = xadd(f.y, pc.ai);
            rescale_out[mode * n_pix + ip] = kmean / fma(er, er, fma(ei, ei, pc.var));
        }
    }
}

// Every float x in [lo, hi] (positive): the largest |lg2.approx(x) - log2(x)|
// / (LG2_EA + LG2_ER |lg2.approx(x)|) into out[0] and the largest absolute
// error into out[1], both as the bit patterns of non-negative doubles.
__global__ void k_log2_error(unsigned lo_bits, unsigned long long count,
                             unsigned long long *__restrict__ out) {
    double worst = 0., wabs = 0.;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         i < count; i += stride) {
        const float x = __uint_as_float(lo_bits + (unsigned)i);
        const float y = lg2_approx(x);
        const double e = fabs((double)y - log2((double)x));
        worst = fmax(worst, e / (LG2_EA + LG2_ER * fabs((double)y)));
        wabs = fmax(wabs, e);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        worst = fmax(worst, __shfl_xor_sync(RSPI_FULL_MASK, worst, o));
        wabs = fmax(wabs, __shfl_xor_sync(RSPI_FULL_MASK, wabs, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], (unsigned long long)__double_as_longlong(worst));
        atomicMax(&out[1], (unsigned long long)__double_as_longlong(wabs));
    }
}

// Per-state sums of the frames' scales, S[s] = sum_{d: fstate[d] = s} scale[d].
__global__ void k_state_scale_sums(const int *__restrict__ fstate, const double *__restrict__ scales,
                                   long long n, long long n_ref, double *__restrict__ ssum,
                                   int *err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        const int s = fstate[d];
        if (s < 0 || s >= n_ref) {
            rspi_flag(err, RSPI_ERR_INDEX);
            continue;
        }
        atomicAdd(&ssum[s], scales[d]);
    }
}

// Polar grid search of the per-pixel NLL (the comparison for the L-BFGS update):
//   NLL_t(F) = sum_s S_s |F + r_s|^2 - sum_s K_t[s] log |F + r_s|^2 (+ const)
// over F = a_j e^{i phi_i}, phi_i = 2 pi i / n_phase, a_j = A (j + 1) / n_amp,
// A = sqrt(sum K / sum S) + max_s |r_s| (every amplitude the data allow).
// The quadratic term is analytic (sum S |F|^2 + 2 Re(conj(F) sum S r) +
// sum S |r|^2); the log term runs over the populated states.  The lowest
// value wins (first candidate index on ties); the pixel's model value and
// its NLL (without the F-independent sum k log s) are written.
constexpr int GR_THREADS = 256;

__global__ void __launch_bounds__(GR_THREADS)
k_grid(double2 *__restrict__ fconv, const int *__restrict__ pixels,
       const int *__restrict__ hist_row, const int *__restrict__ hist, long long n_ref,
       const double *__restrict__ ssum, const double *__restrict__ ref_params, int size,
       int n_phase, int n_amp, double *__restrict__ best_out) {
    __shared__ double fr_re[POP_CAP], fr_im[POP_CAP], fk[POP_CAP];
    __shared__ double scratch[32];
    __shared__ int iscratch[32];
    __shared__ int wsum[32];
    const long long ip = blockIdx.x;
    const int t = pixels[ip];
    const int *hrow = hist + (long long)hist_row[ip] * n_ref;
    PixelConsts pc;
    {
        const double ds = (double)size, c0 = (double)(size / 2);
        const int tx = t / size, ty = t - (t / size) * size;
        pc.qx = ((double)tx - c0) / ds;
        pc.qy = ((double)ty - c0) / ds;
        pc.qrad = sqrt(xadd(xmul(pc.qx, pc.qx), xmul(pc.qy, pc.qy)));
        if (pc.qrad == 0.) pc.qrad = 1.e-6;  // maxLP.py:85
    }
    double st = 0., srr = 0., sri = 0., sq = 0., ks = 0., rmax = 0.;
    for (long long s = threadIdx.x; s < n_ref; s += blockDim.x) {
        const double w = ssum[s];
        ks += (double)hrow[s];
        if (w > 0.) {
            const double2 r = fref_value(pc.qx, pc.qy, pc.qrad, ref_params[3 * s],
                                         ref_params[3 * s + 1], ref_params[3 * s + 2]);
            st += w;
            srr += w * r.x;
            sri += w * r.y;
            sq += w * (r.x * r.x + r.y * r.y);
            rmax = fmax(rmax, hypot(r.x, r.y));
        }
    }
    st = block_sum(st, scratch);
    srr = block_sum(srr, scratch);
    sri = block_sum(sri, scratch);
    sq = block_sum(sq, scratch);
    ks = block_sum(ks, scratch);
    {   // block max of rmax (non-negative: integer order of the bit patterns)
        long long b = __double_as_longlong(rmax);
        for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(RSPI_FULL_MASK, b, o));
        __syncthreads();
        if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = __longlong_as_double(b);
        __syncthreads();
        double m = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, scratch[w]);
        rmax = m;
        __syncthreads();
    }
    if (st == 0.) {   // no frame: the model stays, NLL 0
        if (threadIdx.x == 0) best_out[ip] = 0.;
        return;
    }
    int npop = 0;
    const bool one_chunk = n_ref <= POP_CAP;
    if (one_chunk) load_populated(0, hrow, n_ref, ref_params, pc, fr_re, fr_im, fk, &npop, wsum);
    const double amp = sqrt(ks / st) + rmax;
    const int ncand = n_phase * n_amp;
    double best = -INFINITY;   // maximise -NLL with the shared first-index rule
    int bidx = 0x7fffffff;
    for (int c0 = 0; c0 < ncand; c0 += blockDim.x) {
        const int c = c0 + threadIdx.x;
        const int cc = c < ncand ? c : 0;
        const int i = cc / n_amp, j = cc - (cc / n_amp) * n_amp;
        const double a = amp * (double)(j + 1) / (double)n_amp;
        double sphi, cphi;
        sincos(2. * PI * (double)i / (double)n_phase, &sphi, &cphi);
        const double fx = a * cphi, fy = a * sphi;
        double acc = 0.;
        int s_next = 0;
        do {
            if (!one_chunk)
                s_next = load_populated(s_next, hrow, n_ref, ref_params, pc, fr_re, fr_im, fk,
                                        &npop, wsum);
            else
                s_next = (int)n_ref;
            for (int k = 0; k < npop; ++k) {
                const double re = fx + fr_re[k], im = fy + fr_im[k];
                acc = fma(fk[k], log(re * re + im * im), acc);
            }
            if (!one_chunk) __syncthreads();
        } while (s_next < n_ref);
        const double quad = st * (fx * fx + fy * fy) + 2. * (fx * srr + fy * sri) + sq;
        const double v = -(quad - acc);
        if (c < ncand && argmax_better(v, c, best, bidx)) {
            best = v;
            bidx = c;
        }
    }
    block_argmax(best, bidx, scratch, iscratch);
    if (threadIdx.x == 0) {
        const int i = bidx / n_amp, j = bidx - (bidx / n_amp) * n_amp;
        const double a = amp * (double)(j + 1) / (double)n_amp;
        double sphi, cphi;
        sincos(2. * PI * (double)i / (double)n_phase, &sphi, &cphi);
        fconv[t] = make_double2(a * cphi, a * sphi);
        best_out[ip] = -best;
    }
}

__global__ void __launch_bounds__(1024) k_mean(const double *__restrict__ v, long long n,
                                               double *__restrict__ out) {
    __shared__ double scratch[32];
    double a = 0.;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) a += v[i];
    a = block_sum(a, scratch);
    if (threadIdx.x == 0) *out = a / (double)n;
}

// ---------------------------------------------------------------------------
// Per-pixel, per-frame API of the reference phaser (maxLP.py:107-114,
// 216-253): the photons every frame puts on model pixel t, the frames'
// reference amplitudes there, and per-candidate rescales and log-likelihoods
// over the frames, without the state aggregation of k_pattern.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pixel_q(int t, int size, double &qx, double &qy, double &qrad) {
    const double ds = (double)size, c0 = (double)(size / 2);
    const int tx = t / size, ty = t - (t / size) * size;
    qx = ((double)tx - c0) / ds;
    qy = ((double)ty - c0) / ds;
    qrad = sqrt(xadd(xmul(qx, qx), xmul(qy, qy)));
    if (qrad == 0.) qrad = 1.e-6;  // maxLP.py:85
}

// One warp per listed frame: k = photons of frame d at the detector pixel
// rint(R(-theta_d) q_t size) + size/2 (maxLP.py:250-253),
// fref = ff(pi qrad dia_d) exp(2 pi i q_t . shift_d) (maxLP.py:238-243).
__global__ void k_pixel_frames(int t, int size, const int *__restrict__ d_vals, long long n_vals,
                               const int *__restrict__ ones, const int *__restrict__ multi,
                               const long long *__restrict__ ones_accum,
                               const long long *__restrict__ multi_accum,
                               const int *__restrict__ place_ones,
                               const int *__restrict__ place_multi,
                               const int *__restrict__ count_multi, long long n_data,
                               const double *__restrict__ rot_cs,
                               const double *__restrict__ fparams, double *__restrict__ k_out,
                               double2 *__restrict__ fref_out, int *err) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    double qx, qy, qrad;
    pixel_q(t, size, qx, qy, qrad);
    const int tx = t / size, ty = t - (t / size) * size;
    for (long long i = warp; i < n_vals; i += nwarp) {
        const long long d = d_vals ? (long long)d_vals[i] : i;
        if (d < 0 || d >= n_data) {
            if (lane == 0) {
                rspi_flag(err, RSPI_ERR_INDEX);
                k_out[i] = 0.;
                fref_out[i] = make_double2(0., 0.);
            }
            continue;
        }
        int ox, oy;
        forward_pixel(tx, ty, rot_cs[2 * d], rot_cs[2 * d + 1], size, ox, oy);
        // the flat column x * size + y as the reference's CSR lookup takes it
        // (y == size aliases pixel (x + 1, 0) for even sizes); off the
        // matrix it reads 0
        const long long uf = (long long)ox * size + oy;
        const bool on = uf >= 0 && uf < (long long)size * size;
        const int u = on ? (int)uf : -1;
        long long cnt = 0;
        if (on) {
            const long long oa = ones_accum[d], ma = multi_accum[d];
            for (int j = lane; j < ones[d]; j += 32) cnt += place_ones[oa + j] == u;
            for (int j = lane; j < multi[d]; j += 32)
                if (place_multi[ma + j] == u) cnt += count_multi[ma + j];
        }
        cnt = warp_sum(cnt);
        if (lane == 0) {
            k_out[i] = (double)cnt;
            fref_out[i] = fref_value(qx, qy, qrad, fparams[3 * d], fparams[3 * d + 1],
                                     fparams[3 * d + 2]);
        }
    }
}

// One CTA per candidate f_c over the n frames (maxLP.py:216-228, 181-197):
//   mode 0: rho_c = mean_d k_d / mean_d |f_c + fref_d|^2
//   mode 1: mean_d k_d log(rho |f_c + fref_d|^2) - mean_d rho |f_c + fref_d|^2
//           with rho = rescale_vec[c] (per candidate) or the scalar rescale.
__global__ void __launch_bounds__(256)
k_pixel_values(const double2 *__restrict__ cands, long long n_c, const double *__restrict__ k,
               const double2 *__restrict__ fref, long long n, int mode, double rescale,
               const double *__restrict__ rescale_vec, double *__restrict__ out) {
    __shared__ double scratch[32];
    for (long long c = blockIdx.x; c < n_c; c += gridDim.x) {
        const double2 f = cands[c];
        const double rho = rescale_vec ? rescale_vec[c] : rescale;
        double a = 0., b = 0.;
        for (long long d = threadIdx.x; d < n; d += blockDim.x) {
            const double re = xadd(f.x, fref[d].x), im = xadd(f.y, fref[d].y);
            const double w = xadd(xmul(re, re), xmul(im, im));
            if (mode == 0) {
                a = xadd(a, k[d]);
                b = xadd(b, w);
            } else {
                const double rw = xmul(rho, w);
                a = xadd(a, xmul(k[d], log(rw)));
                b = xadd(b, rw);
            }
        }
        a = block_sum(a, scratch);
        b = block_sum(b, scratch);
        if (threadIdx.x == 0)
            out[c] = mode == 0 ? (a / (double)n) / (b / (double)n)
                               : xsub(a / (double)n, b / (double)n);
    }
}

// Sphere transform ff(pi qrad dia) of every model pixel (maxLP.py:266-269)
// and, with fobj, the holographic amplitude fobj + ff e^{2 pi i q . shift}
// (maxLP.py:260-264).
__global__ void k_fcalc(int size, double dia, double sx, double sy,
                        const double2 *__restrict__ fobj, double *__restrict__ sphere,
                        double2 *__restrict__ fcalc) {
    const long long npix = (long long)size * size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < npix; t += stride) {
        double qx, qy, qrad;
        pixel_q((int)t, size, qx, qy, qrad);
        const double2 r = fref_value(qx, qy, qrad, sx, sy, dia);
        if (sphere) {
            const double sval = xmul(xmul(PI, qrad), dia);
            sphere[t] = xsub(sin(sval), xmul(sval, cos(sval))) / pow(sval, 3.);
        }
        if (fcalc) fcalc[t] = make_double2(xadd(fobj[t].x, r.x), xadd(fobj[t].y, r.y));
    }
}

}  // namespace

extern "C" int rspi_maxlp_frame_params(const int *rmax, long long n_data, long long num_rot,
                                       long long n_ref, int *fstate, int *frot, int *nstate,
                                       int *err, cudaStream_t stream) {
    if (!rmax || !fstate || !frot || !nstate || n_data <= 0 || num_rot <= 0 || n_ref <= 0)
        return RSPI_ERR_ARG;
    cudaMemsetAsync(nstate, 0, sizeof(int) * n_ref, stream);
    k_frame_params<<<rspi_blocks(n_data, 256), 256, 0, stream>>>(rmax, n_data, num_rot, n_ref,
                                                                fstate, frot, nstate, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_histogram(const int *ones, const int *multi,
                                    const long long *ones_accum, const long long *multi_accum,
                                    const int *place_ones, const int *place_multi,
                                    const int *count_multi, long long n_data, const int *fstate,
                                    const int *frot, const double *rot_cs, long long size,
                                    const int *mask_idx, long long n_mask, long long n_ref,
                                    int *hist, int *err, cudaStream_t stream) {
    if (n_data <= 0 || size <= 1 || size > 46340 || n_mask < 0 || n_ref <= 0 || !hist ||
        !mask_idx || !fstate || !frot || !rot_cs)
        return RSPI_ERR_ARG;
    k_histogram<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, n_data,
        fstate, frot, rot_cs, (int)size, mask_idx, n_ref, hist, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_pixel_map(const double *rot_cs, long long num_rot, long long size,
                                    const int *mask_idx, int *cnt, long long *map_off,
                                    int *map_rows, cudaStream_t stream) {
    if (!rot_cs || !mask_idx || !cnt || !map_off || !map_rows || num_rot <= 0 || size <= 1 ||
        size > 46340 || num_rot * size * size > 0x7fffffffLL)
        return RSPI_ERR_ARG;
    const long long n = num_rot * size * size;
    const unsigned grid = rspi_blocks(n, 256);
    cudaMemsetAsync(cnt, 0, sizeof(int) * n, stream);
    k_pixel_map_count<<<grid, 256, 0, stream>>>(rot_cs, num_rot, (int)size, mask_idx, cnt);
    const int st = rspi_scan_rows(cnt, n, map_off, stream);
    if (st != RSPI_OK) return st;
    cudaMemsetAsync(cnt, 0, sizeof(int) * n, stream);
    k_pixel_map_fill<<<grid, 256, 0, stream>>>(rot_cs, num_rot, (int)size, mask_idx, map_off,
                                               cnt, map_rows);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_histogram_map(const int *ones, const int *multi,
                                        const long long *ones_accum, const long long *multi_accum,
                                        const int *place_ones, const int *place_multi,
                                        const int *count_multi, long long n_data,
                                        const int *fstate, const int *frot, long long num_rot,
                                        long long size, const long long *map_off,
                                        const int *map_rows, long long n_ref, int *hist, int *err,
                                        cudaStream_t stream) {
    if (n_data <= 0 || size <= 1 || size > 46340 || num_rot <= 0 || n_ref <= 0 || !hist ||
        !map_off || !map_rows || !fstate || !frot)
        return RSPI_ERR_ARG;
    k_histogram_map<<<rspi_blocks(n_data * 32, 256), 256, 0, stream>>>(
        ones, multi, ones_accum, multi_accum, place_ones, place_multi, count_multi, n_data,
        fstate, frot, num_rot, (int)size, map_off, map_rows, n_ref, hist, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_pattern(double *fconv, const int *pixels, const int *hist_row,
                                  long long n_pix, const int *hist, long long n_ref,
                                  const int *nstate, long long n_modes, const double *ref_params,
                                  long long size, int rescale_mode, const double *rescale,
                                  int num_iter, double *rescale_out, cudaStream_t stream) {
    if (n_pix == 0) return RSPI_OK;  // nothing to search (e.g. an empty ring or mask)
    if (!fconv || !pixels || !hist_row || !hist || !nstate || !ref_params || n_ref <= 0 ||
        n_modes <= 0 || n_modes > 65535 || size <= 1 || size > 46340 || n_pix < 0 ||
        n_pix > 0x7fffffffLL || n_ref * n_modes > 0x7fffffffLL || num_iter < 0 ||
        (rescale_mode == 1 && !rescale) || (rescale_mode != 0 && rescale_mode != 1))
        return RSPI_ERR_ARG;
    const dim3 grid((unsigned)n_pix, (unsigned)n_modes);
    k_pattern<false><<<grid, PT_THREADS, 0, stream>>>(
        (double2 *)fconv, pixels, hist_row, n_pix, hist, n_ref, nstate, n_modes, ref_params,
        (int)size, rescale_mode == 0, rescale, num_iter, rescale_out, nullptr);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_pattern_screened(double *fconv, const int *pixels, const int *hist_row,
                                           long long n_pix, const int *hist, long long n_ref,
                                           const int *nstate, long long n_modes,
                                           const double *ref_params, long long size,
                                           int rescale_mode, const double *rescale, int num_iter,
                                           double *rescale_out, unsigned long long *stats,
                                           cudaStream_t stream) {
    if (n_pix == 0) return RSPI_OK;
    if (!fconv || !pixels || !hist_row || !hist || !nstate || !ref_params || n_ref <= 0 ||
        n_modes <= 0 || n_modes > 65535 || size <= 1 || size > 46340 || n_pix < 0 ||
        n_pix > 0x7fffffffLL || n_ref * n_modes > 0x7fffffffLL || num_iter < 0 ||
        (rescale_mode == 1 && !rescale) || (rescale_mode != 0 && rescale_mode != 1))
        return RSPI_ERR_ARG;
    const dim3 grid((unsigned)n_pix, (unsigned)n_modes);
    k_pattern<true><<<grid, PT_THREADS, 0, stream>>>(
        (double2 *)fconv, pixels, hist_row, n_pix, hist, n_ref, nstate, n_modes, ref_params,
        (int)size, rescale_mode == 0, rescale, num_iter, rescale_out, stats);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_log2_error_max(float lo, float hi, double *out, cudaStream_t stream) {
    if (!out || !(lo > 0.f) || !(hi >= lo) || !(hi < INFINITY)) return RSPI_ERR_ARG;
    unsigned lb, hb;
    memcpy(&lb, &lo, 4);
    memcpy(&hb, &hi, 4);
    cudaMemsetAsync(out, 0, 2 * sizeof(double), stream);
    k_log2_error<<<rspi_sm_count() * 8, 256, 0, stream>>>(
        lb, (unsigned long long)(hb - lb) + 1ull, (unsigned long long *)out);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_mean(const double *vals, long long n, double *out, cudaStream_t stream) {
    if (!vals || !out || n <= 0) return RSPI_ERR_ARG;
    k_mean<<<1, 1024, 0, stream>>>(vals, n, out);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_grid(double *fconv, const int *pixels, const int *hist_row,
                               long long n_pix, const int *hist, long long n_ref,
                               const int *fstate, const double *scales, long long n_data,
                               const double *ref_params, long long size, int n_phase, int n_amp,
                               double *ssum, double *best_nll, int *err, cudaStream_t stream) {
    if (n_pix == 0) return RSPI_OK;
    if (!fconv || !pixels || !hist_row || !hist || !fstate || !scales || !ref_params || !ssum ||
        !best_nll || !err || n_ref <= 0 || n_ref > 0x7fffffffLL || n_data <= 0 || size <= 1 ||
        size > 46340 || n_pix < 0 || n_pix > 0x7fffffffLL || n_phase <= 0 || n_amp <= 0 ||
        (long long)n_phase * n_amp > (1 << 20))
        return RSPI_ERR_ARG;
    cudaMemsetAsync(ssum, 0, sizeof(double) * n_ref, stream);
    k_state_scale_sums<<<rspi_blocks(n_data, 256), 256, 0, stream>>>(fstate, scales, n_data,
                                                                     n_ref, ssum, err);
    k_grid<<<(unsigned)n_pix, GR_THREADS, 0, stream>>>((double2 *)fconv, pixels, hist_row, hist,
                                                       n_ref, ssum, ref_params, (int)size,
                                                       n_phase, n_amp, best_nll);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_pixel_frames(int t, long long size, const int *d_vals, long long n_vals,
                                       const int *ones, const int *multi,
                                       const long long *ones_accum, const long long *multi_accum,
                                       const int *place_ones, const int *place_multi,
                                       const int *count_multi, long long n_data,
                                       const double *rot_cs, const double *fparams,
                                       double *k_out, double *fref_out, int *err,
                                       cudaStream_t stream) {
    if (n_vals == 0) return RSPI_OK;
    if (size <= 1 || size > 46340 || t < 0 || t >= size * size || n_vals < 0 || n_data <= 0 ||
        !ones || !multi || !ones_accum || !multi_accum || !rot_cs || !fparams || !k_out ||
        !fref_out || !err || (!d_vals && n_vals > n_data))
        return RSPI_ERR_ARG;
    k_pixel_frames<<<rspi_blocks(n_vals * 32, 256), 256, 0, stream>>>(
        t, (int)size, d_vals, n_vals, ones, multi, ones_accum, multi_accum, place_ones,
        place_multi, count_multi, n_data, rot_cs, fparams, k_out, (double2 *)fref_out, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_pixel_values(const double *cands, long long n_c, const double *k,
                                       const double *fref, long long n, int mode,
                                       double rescale, const double *rescale_vec, double *out,
                                       cudaStream_t stream) {
    if (n_c == 0) return RSPI_OK;
    if (!cands || !k || !fref || !out || n_c < 0 || n <= 0 || (mode != 0 && mode != 1))
        return RSPI_ERR_ARG;
    const unsigned grid = (unsigned)min(n_c, (long long)rspi_sm_count() * 16);
    k_pixel_values<<<grid, 256, 0, stream>>>((const double2 *)cands, n_c, k,
                                             (const double2 *)fref, n, mode, rescale,
                                             rescale_vec, out);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_maxlp_fcalc(long long size, double dia, double sx, double sy,
                                const double *fobj, double *sphere, double *fcalc,
                                cudaStream_t stream) {
    if (size <= 1 || size > 46340 || (!sphere && !fcalc) || (fcalc && !fobj)) return RSPI_ERR_ARG;
    k_fcalc<<<rspi_blocks(size * size, 256), 256, 0, stream>>>(
        (int)size, dia, sx, sy, (const double2 *)fobj, sphere, (double2 *)fcalc);
    RSPI_RETURN_LAUNCH();
}
