// Dense high-fluence likelihood (row a7 for frames stored as dense uint16):
// the photon term sum_p K[d][p] L[r][p] as a tensor-core GEMM on sm_100a.
//
//   LL[r][d] = init[r / num_rot] * scale[d] + sum_{p in sel} K[d][p] L[r][p]
//
// (calc_prob_all, kernels.cu:116-137, with every pixel of the frame an
// entry).  K is exact in BF16 up to 256 photons, so K = K0 + K1 with
// K0 = K & 255 and K1 = K - K0 (a multiple of 256 below 65536, also exact);
// K1 is only used when some pixel holds more than 255 photons.  The FP64
// log-slice value is split as hi = bf16(L), lo = bf16(L - hi), so
// |L - hi - lo| <= 2^-16 |L|.  Every (digit, part) product is accumulated
// in one FP32 TMEM accumulator by tcgen05.mma (kind::f16, BF16 inputs).
//
// Kernel structure (one 128-frame x 128-row tile per CTA, 4 warps):
//   warp 0 lane 0  TMA producer: A digit tiles and B hi/lo tiles of each
//                  64-pixel k-block into a ring of shared-memory stages
//                  (128-byte swizzle), completion on a "full" mbarrier;
//   warp 1 lane 0  MMA issuer: 4 x (digits x 2) tcgen05.mma per k-block,
//                  tcgen05.commit to the stage's "empty" mbarrier, and a
//                  final commit to the accumulator barrier;
//   all warps      epilogue: tcgen05.ld of its 32 TMEM lanes (frames),
//                  + init * scale, coalesced FP32 stores (frames contiguous).
// Every mbarrier wait is bounded (about one second); on expiry the kernel
// records RSPI_ERR_TIMEOUT, stops issuing, waits (bounded) for what it has
// issued, frees its TMEM and skips the stores.  No cluster multicast.
//
// Exact integer variant (kind::i8): counts K <= 255 as u8 and the log-slice
// in fixed point, Lq = rint(L * 2^21) (|L| < 1024, so Lq fits int32), as
// four 8-bit digits Lq = b3 2^24 + b2 2^16 + b1 2^8 + b0 (b0..b2 unsigned,
// b3 signed).  Each digit product accumulates in its own int32 TMEM
// accumulator, exactly (sum_p K_p * 255 < 2^31 for fewer than 8.4e6 photons
// per frame); the epilogue combines them in FP64, so the only error of
// sum_p K_p L_p is the quantisation, at most 2^-22 sum_p K_p.
#include <cuda.h>
#include <cuda_bf16.h>

#include "rspi_common.cuh"

namespace {

constexpr int DN_BM = 128;          // frames per tile = TMEM lanes
constexpr int DN_BN = 128;          // likelihood rows per tile = TMEM columns (FP32)
constexpr int DN_BK = 64;           // pixels per k-block: 64 x 2 B = one 128-byte swizzle row
constexpr int DN_UK = 16;           // K of one kind::f16 MMA
constexpr int DN_TILE_BYTES = DN_BM * DN_BK * 2;   // 16 KB (A and B tiles alike: 128 x 64)
constexpr int DN_SMEM_BUDGET = 200 * 1024;
constexpr long long DN_WAIT_NS = 1000000000LL;     // bounded waits: 1 s

static_assert(DN_BM == DN_BN, "A and B tiles share one TMA box");

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of parity `parity` to complete; false after DN_WAIT_NS.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > (unsigned long long)DN_WAIT_NS) return false;
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor: K-major tile of 128-byte rows with the
// 128-byte swizzle, 8-row groups 1024 bytes apart (stride byte offset), the
// leading byte offset unused for this layout (encoded 1), descriptor
// version 1 (bits 46-47), swizzle mode 2 = 128B (bits 61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A and B BF16
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
constexpr uint32_t DN_IDESC = (1u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(DN_BN >> 3) << 17) | ((uint32_t)(DN_BM >> 4) << 24);

// kind::i8: D S32 (bits 4-5 = 2), A unsigned 8-bit (bits 7-9 = 0), B
// unsigned or signed 8-bit (bits 10-12 = 0 / 1), K-major, same N/M fields.
constexpr uint32_t DN_IDESC_I8 = (2u << 4) | ((uint32_t)(DN_BN >> 3) << 17) |
                                 ((uint32_t)(DN_BM >> 4) << 24);
constexpr uint32_t DN_IDESC_I8_SB = DN_IDESC_I8 | (1u << 10);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(DN_IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
        "[%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// B operand tiles: BF16 hi, lo (KIND 0) or the four L digits (KIND 1).
struct DenseMaps {
    CUtensorMap a0, a1, b[4];
};

constexpr int KIND_BF16 = 0, KIND_I8 = 1;

// Dynamic shared memory: [stages][A digits + B parts tiles] of 16 KB.
// KIND_BF16: n_digits (1-2) BF16 count digits, B hi/lo, one FP32 accumulator.
// KIND_I8:   one u8 count tile, four L-digit tiles, four int32 accumulators.
template <int KIND>
__global__ void __launch_bounds__(128, 1)
k_dense_ll(const __grid_constant__ DenseMaps maps, int n_digits, int stages, int n_kb,
           long long n_frames, long long row_begin, long long row_end, long long num_rot,
           const double *__restrict__ init, const double *__restrict__ scales,
           float *__restrict__ prob, long long ld, int *err) {
    extern __shared__ uint8_t dn_smem_raw[];
    __shared__ uint64_t bars[2 * 8 + 1];
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_sh;
    constexpr int B_PARTS = KIND == KIND_I8 ? 4 : 2;
    constexpr uint32_t TMEM_COLS = KIND == KIND_I8 ? 4 * DN_BN : DN_BN;
    constexpr int KB_ELEMS = KIND == KIND_I8 ? 128 : DN_BK;   // elements per 128-byte row

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (smem_u32(dn_smem_raw) + 1023u) & ~1023u;
    const int tiles = n_digits + B_PARTS;
    const uint32_t stage_bytes = (uint32_t)tiles * DN_TILE_BYTES;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[8]);
    const uint32_t accb = smem_u32(&bars[16]);
    const long long frame0 = (long long)blockIdx.x * DN_BM;
    const long long rr0 = (long long)blockIdx.y * DN_BN;   // local row of this tile

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(accb, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0 && lane == 0) {
        // producer
        int issued = 0;
        for (int kb = 0; kb < n_kb; ++kb) {
            const int s = kb % stages;
            const uint32_t use = (uint32_t)(kb / stages);
            if (kb >= stages && !mbar_wait(empty0 + 8 * s, (use - 1u) & 1u)) {
                rspi_flag(err, RSPI_ERR_TIMEOUT);
                atomicExch(&abort_sh, 1);
                break;
            }
            if (*(volatile int *)&abort_sh) break;
            const uint32_t st = base + (uint32_t)s * stage_bytes;
            mbar_expect_tx(full0 + 8 * s, stage_bytes);
            const int x = kb * KB_ELEMS;
            tma_load_2d(st, &maps.a0, x, (int)frame0, full0 + 8 * s);
            if (n_digits > 1) tma_load_2d(st + DN_TILE_BYTES, &maps.a1, x, (int)frame0, full0 + 8 * s);
            const uint32_t sb = st + (uint32_t)n_digits * DN_TILE_BYTES;
#pragma unroll
            for (int part = 0; part < B_PARTS; ++part)
                tma_load_2d(sb + (uint32_t)part * DN_TILE_BYTES, &maps.b[part], x, (int)rr0,
                            full0 + 8 * s);
            ++issued;
        }
        // every issued load lands before the CTA can exit
        for (int kb = (issued > stages ? issued - stages : 0); kb < issued; ++kb)
            if (!mbar_wait(full0 + 8 * (kb % stages), (uint32_t)(kb / stages) & 1u)) {
                rspi_flag(err, RSPI_ERR_TIMEOUT);
                atomicExch(&abort_sh, 1);
            }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        for (int kb = 0; kb < n_kb; ++kb) {
            const int s = kb % stages;
            if (*(volatile int *)&abort_sh) break;
            if (!mbar_wait(full0 + 8 * s, (uint32_t)(kb / stages) & 1u)) {
                rspi_flag(err, RSPI_ERR_TIMEOUT);
                atomicExch(&abort_sh, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + (uint32_t)s * stage_bytes;
            const uint32_t sb = st + (uint32_t)n_digits * DN_TILE_BYTES;
            // 4 MMAs of 32 bytes of K per 128-byte row (16 BF16 or 32 int8 elements)
            if (KIND == KIND_I8) {
#pragma unroll
                for (int part = 0; part < 4; ++part)
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint32_t koff = (uint32_t)k * 32;
                        const uint64_t ad = sw128_desc(st + koff);
                        const uint64_t bd = sw128_desc(sb + (uint32_t)part * DN_TILE_BYTES + koff);
                        mma_i8(tmem + (uint32_t)part * DN_BN, ad, bd,
                               part == 3 ? DN_IDESC_I8_SB : DN_IDESC_I8, (kb | k) != 0);
                    }
            } else {
                for (int dg = 0; dg < n_digits; ++dg)
                    for (int part = 0; part < 2; ++part)
#pragma unroll
                        for (int k = 0; k < DN_BK / DN_UK; ++k) {
                            const uint32_t koff = (uint32_t)k * DN_UK * 2;
                            const uint64_t ad =
                                sw128_desc(st + (uint32_t)dg * DN_TILE_BYTES + koff);
                            const uint64_t bd =
                                sw128_desc(sb + (uint32_t)part * DN_TILE_BYTES + koff);
                            mma_bf16(tmem, ad, bd, (kb | dg | part | k) != 0);
                        }
            }
            mma_commit(empty0 + 8 * s);
        }
        mma_commit(accb);   // arrives once every MMA issued above has completed
    }
    __syncwarp();

    // epilogue: TMEM lanes 32*warp .. +31 are frames frame0 + 32*warp + lane
    const bool ready = mbar_wait(accb, 0);
    if (!ready) rspi_flag(err, RSPI_ERR_TIMEOUT);
    // one decision for the whole CTA (tcgen05.ld is warp-collective)
    const bool ok = __syncthreads_and(ready && !abort_sh) && n_kb > 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const long long d = frame0 + 32 * warp + lane;
    const double sc = d < n_frames ? scales[d] : 0.;
    if (ok) {
        const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
        for (int c0 = 0; c0 < DN_BN; c0 += 32) {
            double acc[32];
            if (KIND == KIND_I8) {
                // sum_j 2^(8j) C_j, then the fixed-point scale 2^-21 (exact in FP64
                // up to the final rounding of the four-term sum)
                float v[32];
                tmem_ld32(lane_base + 3u * DN_BN + (uint32_t)c0, v);
#pragma unroll
                for (int j = 0; j < 32; ++j) acc[j] = (double)__float_as_int(v[j]);
                for (int part = 2; part >= 0; --part) {
                    tmem_ld32(lane_base + (uint32_t)part * DN_BN + (uint32_t)c0, v);
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        acc[j] = fma(acc[j], 256., (double)__float_as_int(v[j]));
                }
#pragma unroll
                for (int j = 0; j < 32; ++j) acc[j] *= 4.76837158203125e-07;   // 2^-21
            } else {
                float v[32];
                tmem_ld32(lane_base + (uint32_t)c0, v);
#pragma unroll
                for (int j = 0; j < 32; ++j) acc[j] = (double)v[j];
            }
            if (d < n_frames) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const long long rr = rr0 + c0 + j;
                    const long long r = row_begin + rr;
                    if (r < row_end)
                        prob[rr * ld + d] = (float)(init[r / num_rot] * sc + acc[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
}

// Dense frames -> BF16 digit matrices over the likelihood pixels (K-major,
// k_pad columns, zero beyond n_sel); kmax gets the largest count seen.
__global__ void k_dense_frames(const unsigned short *__restrict__ frames, long long n_frames,
                               long long npix, const int *__restrict__ sel_pix, long long n_sel,
                               long long k_pad, __nv_bfloat16 *__restrict__ a0,
                               __nv_bfloat16 *__restrict__ a1, int *__restrict__ kmax) {
    const long long total = n_frames * k_pad;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int mx = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long d = i / k_pad, c = i - d * k_pad;
        const int k = c < n_sel ? (int)frames[d * npix + sel_pix[c]] : 0;
        mx = max(mx, k);
        a0[i] = __int2bfloat16_rn(k & 255);
        if (a1) a1[i] = __int2bfloat16_rn(k & ~255);
    }
    mx = warp_max_int(mx);
    if ((threadIdx.x & 31) == 0) atomicMax(kmax, mx);
}

// Rotated log-slices split into BF16 hi + lo parts (same values as
// k_rot_log_js: rot_log_value in FP64), zero beyond n_sel.
__global__ void __launch_bounds__(256)
k_rot_log_split(const double *__restrict__ holo, long long num_rot,
                const double *__restrict__ rot_cs, int size, const double *__restrict__ bg,
                const int *__restrict__ sel_pix, long long n_sel, long long k_pad,
                long long row_begin, long long n_rows, __nv_bfloat16 *__restrict__ hi,
                __nv_bfloat16 *__restrict__ lo, float *__restrict__ abs_max) {
    const long long npix = (long long)size * size;
    const int ns = (int)n_sel, kp = (int)k_pad;
    float amax = 0.f;
    const float inv_size = 1.f / (float)size;
    for (long long rr = blockIdx.x; rr < n_rows; rr += gridDim.x) {   // one row per CTA
        const long long r = row_begin + rr;
        const long long s0 = r / num_rot, j = r - s0 * num_rot;
        const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
        const double *w = holo + s0 * npix;
        for (int c = threadIdx.x; c < kp; c += blockDim.x) {
            double v = 0.;
            if (c < ns) {
                const int p = sel_pix[c];
                int x, y;
                pixel_xy(p, size, inv_size, x, y);
                v = rot_log_value(w, x, y, size, ac, as, bg[p]);
            }
            const __nv_bfloat16 h = __double2bfloat16(v);
            const long long i = rr * k_pad + c;
            hi[i] = h;
            lo[i] = __double2bfloat16(v - (double)__bfloat162float(h));
            amax = fmaxf(amax, fabsf((float)v));
        }
    }
    if (abs_max) {
        amax = __int_as_float(warp_max_int(__float_as_int(amax)));
        if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(abs_max), __float_as_int(amax));
    }
}

// Dense frames -> u8 counts over the likelihood pixels (kmax: largest count,
// the caller checks it is below 256).
__global__ void k_dense_frames_u8(const unsigned short *__restrict__ frames, long long n_frames,
                                  long long npix, const int *__restrict__ sel_pix,
                                  long long n_sel, long long k_pad, uint8_t *__restrict__ a,
                                  int *__restrict__ kmax) {
    const long long total = n_frames * k_pad;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int mx = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long d = i / k_pad, c = i - d * k_pad;
        const int k = c < n_sel ? (int)frames[d * npix + sel_pix[c]] : 0;
        mx = max(mx, k);
        a[i] = (uint8_t)min(k, 255);
    }
    mx = warp_max_int(mx);
    if ((threadIdx.x & 31) == 0) atomicMax(kmax, mx);
}

// Rotated log-slices (rot_log_value, FP64) in fixed point Lq = rint(L 2^21)
// as four 8-bit digit planes b[part][row][c] (zero beyond n_sel).  |L| is
// below 1024 for every value rot_log_value returns (the -1000 sentinel, and
// logs of doubles); a larger value is clamped and flagged.
__global__ void __launch_bounds__(256)
k_rot_log_q(const double *__restrict__ holo, long long num_rot, const double *__restrict__ rot_cs,
            int size, const double *__restrict__ bg, const int *__restrict__ sel_pix,
            long long n_sel, long long k_pad, long long row_begin, long long n_rows,
            long long plane, uint8_t *__restrict__ b, int *err) {
    const long long npix = (long long)size * size;
    const int ns = (int)n_sel, kp = (int)k_pad;
    const float inv_size = 1.f / (float)size;
    for (long long rr = blockIdx.x; rr < n_rows; rr += gridDim.x) {   // one row per CTA
        const long long r = row_begin + rr;
        const long long s0 = r / num_rot, j = r - s0 * num_rot;
        const double ac = rot_cs[2 * j], as = rot_cs[2 * j + 1];
        const double *w = holo + s0 * npix;
        uint8_t *o = b + rr * k_pad;
        // four consecutive columns per thread: one 32-bit store per digit plane
        for (int c0 = 4 * threadIdx.x; c0 < kp; c0 += 4 * blockDim.x) {
            uint32_t dg[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int c = c0 + u;
                double v = 0.;
                if (c < ns) {
                    const int p = sel_pix[c];
                    int x, y;
                    pixel_xy(p, size, inv_size, x, y);
                    v = rot_log_value(w, x, y, size, ac, as, bg[p]);
                }
                if (!(fabs(v) < 1023.)) {   // also NaN
                    rspi_flag(err, RSPI_ERR_CAPACITY);
                    v = v != v ? 0. : (v > 0. ? 1023. : -1023.);
                }
                const uint32_t q = (uint32_t)__double2int_rn(v * 2097152.);   // rint(v 2^21)
#pragma unroll
                for (int d = 0; d < 4; ++d) dg[d] |= ((q >> (8 * d)) & 255u) << (8 * u);
            }
#pragma unroll
            for (int d = 0; d < 4; ++d)
                *reinterpret_cast<uint32_t *>(o + (long long)d * plane + c0) = dg[d];
        }
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 2-D map over a rows x k_pad K-major matrix of BF16 (64 x 128 boxes) or
// 8-bit (128 x 128 boxes) elements: 128-byte box rows, 128B swizzle, zero
// fill outside (rows beyond the matrix read as zeros).
bool make_map(CUtensorMap *m, const void *ptr, long long k_pad, long long rows, bool byte) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int esz = byte ? 1 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)k_pad * esz};
    cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)DN_BM};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, byte ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
              const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int KIND>
int launch_dense(const DenseMaps &maps, int n_digits, long long k_pad, long long n_frames,
                 long long n_rows, long long num_rot, long long row_begin, long long row_end,
                 const double *init, const double *scales, float *prob, long long ld, int *err,
                 cudaStream_t stream) {
    const int b_parts = KIND == KIND_I8 ? 4 : 2;
    const int stage_bytes = (n_digits + b_parts) * DN_TILE_BYTES;
    const int stages = min(8, DN_SMEM_BUDGET / stage_bytes);
    const int smem = stages * stage_bytes + 1024;
    static RspiSmemOptIn optin;
    if (!rspi_smem_optin((const void *)k_dense_ll<KIND>, DN_SMEM_BUDGET + 1024, optin))
        return RSPI_ERR_CUDA;
    // a launch covers at most 65535 row tiles of 128 rows: larger row ranges
    // are the caller's to split (bad argument)
    if ((n_rows + DN_BN - 1) / DN_BN > 65535) return RSPI_ERR_ARG;
    const dim3 grid((unsigned)((n_frames + DN_BM - 1) / DN_BM),
                    (unsigned)((n_rows + DN_BN - 1) / DN_BN));
    const int n_kb = (int)(k_pad / (KIND == KIND_I8 ? 128 : DN_BK));
    k_dense_ll<KIND><<<grid, 128, smem, stream>>>(maps, n_digits, stages, n_kb, n_frames,
                                                  row_begin, row_end, num_rot, init, scales,
                                                  prob, ld, err);
    RSPI_RETURN_LAUNCH();
}

}  // namespace

extern "C" int rspi_dense_frames(const unsigned short *frames, long long n_frames, long long npix,
                                 const int *sel_pix, long long n_sel, long long k_pad, void *a0,
                                 void *a1, int *kmax, cudaStream_t stream) {
    if (!frames || !sel_pix || !a0 || !kmax || n_frames <= 0 || npix <= 0 || n_sel < 0 ||
        k_pad < n_sel || k_pad % DN_BK)
        return RSPI_ERR_ARG;
    k_dense_frames<<<rspi_blocks(n_frames * k_pad, 256, 16), 256, 0, stream>>>(
        frames, n_frames, npix, sel_pix, n_sel, k_pad, (__nv_bfloat16 *)a0, (__nv_bfloat16 *)a1,
        kmax);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rot_log_split(const double *holo, long long n_states0, long long num_rot,
                                  const double *rot_cs, long long size, const double *bg,
                                  const int *sel_pix, long long n_sel, long long k_pad,
                                  long long row_begin, long long row_end, void *hi, void *lo,
                                  float *abs_max, cudaStream_t stream) {
    if (n_states0 <= 0 || num_rot <= 0 || size <= 1 || size > 46340 || k_pad < n_sel ||
        k_pad % DN_BK || row_begin < 0 || row_end > n_states0 * num_rot || row_end < row_begin ||
        !holo || !rot_cs || !bg || !hi || !lo)
        return RSPI_ERR_ARG;
    const long long n_rows = row_end - row_begin;
    if (n_rows == 0) return RSPI_OK;
    k_rot_log_split<<<(unsigned)min(n_rows, (long long)rspi_sm_count() * 64), 256, 0, stream>>>(
        holo, num_rot, rot_cs, (int)size, bg, sel_pix, n_sel, k_pad, row_begin, n_rows,
        (__nv_bfloat16 *)hi, (__nv_bfloat16 *)lo, abs_max);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_dense_loglike(const void *a0, const void *a1, const void *b_hi,
                                  const void *b_lo, long long k_pad, long long n_frames,
                                  long long n_brows, long long num_rot, long long row_begin,
                                  long long row_end, const double *init, const double *scales,
                                  float *prob, long long ld, int *err, cudaStream_t stream) {
    if (!a0 || !b_hi || !b_lo || !init || !scales || !prob || !err || k_pad <= 0 ||
        k_pad % DN_BK || n_frames <= 0 || num_rot <= 0 || row_begin < 0 ||
        row_end < row_begin || row_end - row_begin > n_brows || ld < n_frames ||
        n_frames > 0x7fffffffLL || n_brows > 0x7fffffffLL || k_pad > 0x7fffffffLL)
        return RSPI_ERR_ARG;
    // TMA: 16-byte aligned bases and row strides (k_pad * 2 bytes, k_pad % 64 == 0)
    const uintptr_t al = (uintptr_t)a0 | (uintptr_t)b_hi | (uintptr_t)b_lo | (uintptr_t)a1;
    if (al & 15) return RSPI_ERR_ARG;
    const long long n_rows = row_end - row_begin;
    if (n_rows == 0) return RSPI_OK;
    const int n_digits = a1 ? 2 : 1;
    DenseMaps maps;
    if (!make_map(&maps.a0, a0, k_pad, n_frames, false) ||
        !make_map(&maps.a1, a1 ? a1 : a0, k_pad, n_frames, false) ||
        !make_map(&maps.b[0], b_hi, k_pad, n_brows, false) ||
        !make_map(&maps.b[1], b_lo, k_pad, n_brows, false))
        return RSPI_ERR_CUDA;
    maps.b[2] = maps.b[0];
    maps.b[3] = maps.b[1];
    return launch_dense<KIND_BF16>(maps, n_digits, k_pad, n_frames, n_rows, num_rot, row_begin,
                                   row_end, init, scales, prob, ld, err, stream);
}

extern "C" int rspi_dense_frames_u8(const unsigned short *frames, long long n_frames,
                                    long long npix, const int *sel_pix, long long n_sel,
                                    long long k_pad, void *a, int *kmax, cudaStream_t stream) {
    if (!frames || !sel_pix || !a || !kmax || n_frames <= 0 || npix <= 0 || n_sel < 0 ||
        k_pad < n_sel || k_pad % 128)
        return RSPI_ERR_ARG;
    k_dense_frames_u8<<<rspi_blocks(n_frames * k_pad, 256, 16), 256, 0, stream>>>(
        frames, n_frames, npix, sel_pix, n_sel, k_pad, (uint8_t *)a, kmax);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_rot_log_fixed(const double *holo, long long n_states0, long long num_rot,
                                  const double *rot_cs, long long size, const double *bg,
                                  const int *sel_pix, long long n_sel, long long k_pad,
                                  long long row_begin, long long row_end, long long plane_rows,
                                  void *digits, int *err, cudaStream_t stream) {
    if (n_states0 <= 0 || num_rot <= 0 || size <= 1 || size > 46340 || k_pad < n_sel ||
        k_pad % 128 || row_begin < 0 || row_end > n_states0 * num_rot || row_end < row_begin ||
        plane_rows < row_end - row_begin || !holo || !rot_cs || !bg || !digits || !err ||
        (reinterpret_cast<uintptr_t>(digits) & 3) != 0)
        return RSPI_ERR_ARG;
    const long long n_rows = row_end - row_begin;
    if (n_rows == 0) return RSPI_OK;
    k_rot_log_q<<<(unsigned)min(n_rows, (long long)rspi_sm_count() * 64), 256, 0, stream>>>(
        holo, num_rot, rot_cs, (int)size, bg, sel_pix, n_sel, k_pad, row_begin, n_rows,
        plane_rows * k_pad, (uint8_t *)digits, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_dense_loglike_i8(const void *a, const void *digits, long long k_pad,
                                     long long n_frames, long long n_brows, long long num_rot,
                                     long long row_begin, long long row_end, const double *init,
                                     const double *scales, float *prob, long long ld, int *err,
                                     cudaStream_t stream) {
    if (!a || !digits || !init || !scales || !prob || !err || k_pad <= 0 || k_pad % 128 ||
        n_frames <= 0 || num_rot <= 0 || row_begin < 0 || row_end < row_begin ||
        row_end - row_begin > n_brows || ld < n_frames || n_frames > 0x7fffffffLL ||
        n_brows > 0x7fffffffLL || k_pad > 0x7fffffffLL)
        return RSPI_ERR_ARG;
    if (((uintptr_t)a | (uintptr_t)digits) & 15) return RSPI_ERR_ARG;
    const long long n_rows = row_end - row_begin;
    if (n_rows == 0) return RSPI_OK;
    const long long plane = n_brows * k_pad;   // bytes per digit plane
    if (plane % 16) return RSPI_ERR_ARG;
    DenseMaps maps;
    if (!make_map(&maps.a0, a, k_pad, n_frames, true)) return RSPI_ERR_CUDA;
    maps.a1 = maps.a0;
    for (int part = 0; part < 4; ++part)
        if (!make_map(&maps.b[part], (const uint8_t *)digits + part * plane, k_pad, n_brows, true))
            return RSPI_ERR_CUDA;
    return launch_dense<KIND_I8>(maps, 1, k_pad, n_frames, n_rows, num_rot, row_begin, row_end,
                                 init, scales, prob, ld, err, stream);
}
