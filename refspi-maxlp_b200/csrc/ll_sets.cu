// Screening likelihood, frame-set form (row a7, the FP32 screening pass of the
// chosen form).
//
// LL32[r][d] = float(init[r / num_rot] * scales[d] + sum over frame d's
// in-mask photons p of L_r(p)) for every likelihood row r (kernels.cu:116-137
// with the slices and sums in FP32; the candidates are rescored in FP64
// afterwards, screen.cu).
//
// Work split.  A CTA takes four consecutive likelihood rows at a time (a
// "tile"); their FP32 slices sit in shared memory interleaved by column,
// tile[c] = (row 0..3 at column c), so one 16-byte gather brings a photon's
// value in all four rows.  Four FP32 rows of a 185^2 detector's likelihood
// columns do not fit in shared memory, so the columns are cut into n_parts
// parts of part_w columns, each copied in with one bulk (TMA) copy from a
// global layout that already holds the tile's four rows interleaved part by
// part (rspi_rot_log_slices_sets).  Eight zero columns follow each part.
//
// Frames are taken 32 at a time ("sets"): lane l of a warp owns frame
// set_frames[32 s + l] and accumulates its four rows alone, so there is no
// cross-lane reduction; the set's results go to likelihood column 32 s + l
// (the caller's frame order, sorted by photon count, defines the columns).
// A 16-byte shared gather is served eight lanes (a quarter warp) per
// wavefront and is conflict-free when the eight addresses fall in the eight
// 16-byte bank groups, i.e. have distinct columns mod 8 ("classes").  Each
// quarter warp's eight frames therefore follow a schedule of steps in which
// the eight lanes always read eight distinct classes: the 8 x 8 matrix of
// (frame, class) photon counts of the part, padded with zero-column reads to
// a regular matrix (every row and column summing to the set's step count),
// is decomposed into permutations (Birkhoff-von Neumann; each permutation is
// a perfect matching of the matrix's support, found by augmenting paths).
// By Koenig's theorem the step count max(largest frame, largest class total)
// is the fewest possible.  Entries: 16-bit local columns, four steps of a
// lane per 8-byte group, groups of a (set, part) in one range (part-major).
#include "rspi_common.cuh"

namespace {

constexpr int SMEM_LIMIT = 227 * 1024;
constexpr int SETS_MAX_PARTS = 4;
constexpr int SETS_MAX_PERMS = 64;   // terms of one decomposition (each zeroes a cell)
constexpr int BUILD_WARPS = 4;
constexpr long long WAIT_NS = 1000000000LL;   // bound of every mbarrier wait (1 s)

__device__ __forceinline__ unsigned entry16_at(const unsigned short *__restrict__ ent16,
                                               long long rr, int lane) {
    return ent16[(rr >> 1) * 64 + lane * 2 + (rr & 1)];
}

// ---------------------------------------------------------------------------
// entry construction (once per dataset and geometry)
// ---------------------------------------------------------------------------

// counts[d * 32 + h * 8 + c]: frame d's photons in part h of local class c.
__global__ void __launch_bounds__(BUILD_WARPS * 32)
k_sets_counts(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
              long long n, int p_zero, int n_parts, int part_w, int *__restrict__ counts) {
    __shared__ int cnt[BUILD_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long d = warp; d < n; d += nwarp) {
        cnt[w][lane] = 0;
        __syncwarp();
        const long long r0 = row_off16[d], nr = row_off16[d + 1] - r0;
        for (long long r = 0; r < nr; ++r) {
            const unsigned e = entry16_at(ent16, r0 + r, lane);
            int key = 32;
            if (e < (unsigned)p_zero) {
                const int h = (int)(e / (unsigned)part_w);
                key = h * 8 + (int)((e - (unsigned)(h * part_w)) & 7u);
            }
            const unsigned m = __match_any_sync(RSPI_FULL_MASK, key);
            if (key < 32 && lane == __ffs(m) - 1) cnt[w][key] += __popc(m);
            __syncwarp();
        }
        counts[d * 32 + lane] = lane < n_parts * 8 ? cnt[w][lane] : 0;
        __syncwarp();
    }
}

// quarter_groups[(h * n_sets + s) * 4 + p] = ceil(D_p / 4), D_p = max(largest
// frame total, largest class total) of quarter warp p of set s in part h;
// groups[h * n_sets + s] = the largest of the four.
__global__ void k_sets_steps(const int *__restrict__ counts, const int *__restrict__ set_frames,
                             long long n_sets, int n_parts, int *__restrict__ groups,
                             int *__restrict__ quarter_groups) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_sets * n_parts;
         i += stride) {
        const int h = (int)(i / n_sets);
        const long long s = i - (long long)h * n_sets;
        int gmax = 0;
        for (int p = 0; p < 4; ++p) {
            int col[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            int dq = 0;
            for (int f = 0; f < 8; ++f) {
                const int d = set_frames[s * 32 + 8 * p + f];
                if (d < 0) continue;
                int row = 0;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int v = counts[(long long)d * 32 + h * 8 + c];
                    row += v;
                    col[c] += v;
                }
                dq = max(dq, row);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) dq = max(dq, col[c]);
            const int gq = (dq + 3) / 4;
            if (quarter_groups) quarter_groups[i * 4 + p] = gq;
            gmax = max(gmax, gq);
        }
        groups[i] = gmax;
    }
}

// ---------------------------------------------------------------------------
// frame grouping: which eight frames share a quarter warp
// ---------------------------------------------------------------------------
// A quarter warp's steps are max(largest frame, largest class total) per
// part, and its gathers cost that many wavefronts whatever its photons.
// With eight frames of alike length taken in rank order the class totals of
// a 250-photon frame's quarter exceed their mean by ~12% (Poisson spread of
// eight frames' photons over eight classes).  So frames are grouped per
// window of GROUP_W frames of neighbouring ranks (sorted by photon count):
//  1. greedy: each quarter starts from the longest frame left and takes, seven
//     times, the frame that keeps sum over parts of max(largest frame,
//     largest class total) smallest (ties: the lower rank);
//  2. pair sweeps: for every pair of quarters (a < b) the best of the 64
//     exchanges of one frame of a with one of b (an empty slot counts as a
//     frame without photons) is made when it lowers the pair's total cost
//     (ties: the lower exchange index), until a sweep changes nothing or
//     `sweeps` are done;
//  3. the window's quarters in decreasing cost (ties: lower index), four to a
//     set, so a set's quarters need alike step counts.
// Everything is integer and in a fixed order: the result is deterministic.
constexpr int GROUP_W = 256;             // frames per window (a multiple of 32)
constexpr int GROUP_Q = GROUP_W / 8;     // quarters per window
constexpr int GROUP_STRIDE = SETS_MAX_PARTS * 8 + 1;
constexpr unsigned long long GROUP_NONE = ~0ull;

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v,
                                                            unsigned long long *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(RSPI_FULL_MASK, v, o);
        v = u < v ? u : v;
    }
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    unsigned long long m = GROUP_NONE;
    for (int k = 0; k < nw; ++k) m = red[k] < m ? red[k] : m;
    return m;
}

// cost of quarter q with slot `slot` holding local frame `f` instead (slot
// -1: as it is): sum over parts of max(largest frame, largest class total)
__device__ __forceinline__ int group_cost(short (*qf)[8], int q, int slot, int f,
                                          int (*cnt)[GROUP_STRIDE], int (*len)[SETS_MAX_PARTS],
                                          int n_parts) {
    int cost = 0;
    for (int p = 0; p < n_parts; ++p) {
        int lane = 0, cls[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            const int g = k == slot ? f : qf[q][k];
            if (g < 0) continue;
            lane = max(lane, len[g][p]);
#pragma unroll
            for (int c = 0; c < 8; ++c) cls[c] += cnt[g][p * 8 + c];
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) lane = max(lane, cls[c]);
        cost += lane;
    }
    return cost;
}

__global__ void __launch_bounds__(GROUP_W)
k_sets_group(const int *__restrict__ counts, const int *__restrict__ order, long long n,
             int n_parts, int sweeps, int *__restrict__ set_frames, int *err) {
    __shared__ int cnt[GROUP_W][GROUP_STRIDE];
    __shared__ int len[GROUP_W][SETS_MAX_PARTS];
    __shared__ short qf[GROUP_Q][8];
    __shared__ int qc[GROUP_Q];
    __shared__ int S[SETS_MAX_PARTS * 8], L[SETS_MAX_PARTS];
    __shared__ unsigned char used[GROUP_W];
    __shared__ unsigned long long red[GROUP_W / 32];
    __shared__ int changed;
    const int t = threadIdx.x;
    const long long w0 = (long long)blockIdx.x * GROUP_W;
    const int m = (int)min((long long)GROUP_W, n - w0);
    const int nq = (m + 7) / 8;
    const int p8 = n_parts * 8;
    // a frame index outside [0, n) is flagged and taken as a frame without
    // photons (its slot is written as -1)
    __shared__ int fid[GROUP_W];
    if (t < m) {
        const int d = order[w0 + t];
        const bool ok = d >= 0 && d < n;
        if (!ok) rspi_flag(err, RSPI_ERR_INDEX);
        fid[t] = ok ? d : -1;
    } else {
        fid[t] = -1;
    }
    __syncthreads();
    for (int i = t; i < GROUP_W * 32; i += blockDim.x) {
        const int f = i >> 5, k = i & 31;
        cnt[f][k] = (f < m && k < p8 && fid[f] >= 0) ? counts[(long long)fid[f] * 32 + k] : 0;
    }
    __syncthreads();
    used[t] = t >= m;
    for (int p = 0; p < SETS_MAX_PARTS; ++p) {
        int s = 0;
        for (int c = 0; c < 8; ++c) s += cnt[t][p * 8 + c];
        len[t][p] = s;
    }
    for (int i = t; i < GROUP_Q * 8; i += blockDim.x) qf[i >> 3][i & 7] = -1;
    __syncthreads();

    // 1. greedy quarters
    for (int q = 0; q < nq; ++q) {
        const unsigned long long seed = block_min_u64(used[t] ? GROUP_NONE : (unsigned long long)t, red);
        if (seed == GROUP_NONE) break;   // uniform; never before the last quarter
        if (t == 0) {
            const int f = (int)seed;
            qf[q][0] = (short)f;
            used[f] = 1;
            for (int k = 0; k < p8; ++k) S[k] = cnt[f][k];
            for (int p = 0; p < n_parts; ++p) L[p] = len[f][p];
        }
        __syncthreads();
        for (int k = 1; k < 8; ++k) {
            unsigned long long key = GROUP_NONE;
            if (!used[t]) {
                int cost = 0;
                for (int p = 0; p < n_parts; ++p) {
                    int v = max(L[p], len[t][p]);
#pragma unroll
                    for (int c = 0; c < 8; ++c) v = max(v, S[p * 8 + c] + cnt[t][p * 8 + c]);
                    cost += v;
                }
                key = ((unsigned long long)(unsigned)cost << 32) | (unsigned)t;
            }
            const unsigned long long best = block_min_u64(key, red);
            if (best == GROUP_NONE) break;   // uniform: every thread saw the same minimum
            if (t == 0) {
                const int f = (int)(best & 0xffffffffu);
                qf[q][k] = (short)f;
                used[f] = 1;
                for (int j = 0; j < p8; ++j) S[j] += cnt[f][j];
                for (int p = 0; p < n_parts; ++p) L[p] = max(L[p], len[f][p]);
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (t < nq) qc[t] = group_cost(qf, t, -1, -1, cnt, len, n_parts);
    __syncthreads();

    // 2. pair sweeps
    for (int sw = 0; sw < sweeps; ++sw) {
        if (t == 0) changed = 0;
        __syncthreads();
        for (int a = 0; a < nq; ++a) {
            for (int b = a + 1; b < nq; ++b) {
                unsigned long long key = GROUP_NONE;
                int ca = 0, cb = 0;
                if (t < 64) {
                    const int i = t >> 3, j = t & 7;
                    const int fa = qf[a][i], fb = qf[b][j];
                    if (fa >= 0 || fb >= 0) {
                        ca = group_cost(qf, a, i, fb, cnt, len, n_parts);
                        cb = group_cost(qf, b, j, fa, cnt, len, n_parts);
                        const int delta = ca + cb - qc[a] - qc[b];
                        // order-preserving map of the signed delta to 32 bits
                        if (delta < 0)
                            key = ((unsigned long long)((unsigned)delta ^ 0x80000000u) << 32) |
                                  (unsigned)t;
                    }
                }
                const unsigned long long best = block_min_u64(key, red);
                if (best != GROUP_NONE && t == (int)(best & 0xffffffffu)) {
                    const int i = t >> 3, j = t & 7;
                    const short fa = qf[a][i];
                    qf[a][i] = qf[b][j];
                    qf[b][j] = fa;
                    qc[a] = ca;
                    qc[b] = cb;
                    changed = 1;
                }
                __syncthreads();
            }
        }
        if (!changed) break;   // uniform: read after the last pair's barrier
        __syncthreads();
    }

    // 3. quarters in decreasing cost, four to a set
    const long long set0 = w0 / 32;
    const int ns = (nq + 3) / 4;
    if (t < nq) {
        int rank = 0;
        for (int q = 0; q < nq; ++q) rank += qc[q] > qc[t] || (qc[q] == qc[t] && q < t);
        for (int k = 0; k < 8; ++k) {
            const int f = qf[t][k];
            set_frames[set0 * 32 + rank * 8 + k] = f >= 0 ? fid[f] : -1;
        }
    }
    for (int i = nq * 8 + t; i < ns * 32; i += blockDim.x) set_frames[set0 * 32 + i] = -1;
}

// Perfect matching of the support of m (8 x 8, m[f][c] > 0) by augmenting
// paths (breadth-first from each row); col_of[f] receives row f's column.
// False when none exists (never, for a regular matrix: Hall's condition).
__device__ bool perfect_matching(const int (&m)[8][8], int (&col_of)[8]) {
    int row_of[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) col_of[k] = row_of[k] = -1;
    for (int f = 0; f < 8; ++f) {
        int prev[8], queue[8];
        for (int c = 0; c < 8; ++c) prev[c] = -1;
        int qh = 0, qt = 0, found = -1;
        unsigned seen = 1u << f;
        queue[qt++] = f;
        while (qh < qt && found < 0) {
            const int r = queue[qh++];
            for (int c = 0; c < 8; ++c) {
                if (m[r][c] <= 0 || prev[c] >= 0) continue;
                prev[c] = r;
                if (row_of[c] < 0) {
                    found = c;
                    break;
                }
                const int r2 = row_of[c];
                if (!((seen >> r2) & 1u)) {
                    seen |= 1u << r2;
                    queue[qt++] = r2;
                }
            }
        }
        if (found < 0) return false;
        // flip the path found -> ... -> f
        int c = found;
        for (int guard = 0; guard < 9; ++guard) {
            const int r = prev[c];
            const int old = col_of[r];
            col_of[r] = c;
            row_of[c] = r;
            if (r == f) break;
            c = old;
        }
    }
    return true;
}

// One warp per (set, part).  Lane 8 p of the warp decomposes quarter warp
// p's count matrix, padded to a regular matrix of its own step count D_p
// (the larger of its fullest frame and its fullest class), into
// permutations (shared memory: packed classes of the eight lanes, 3 bits
// each in 4-bit fields, the multiplicity and the first step of each); then
// every lane places its frame's photons of the part, the k-th photon of
// class c at the k-th step in which the lane reads class c, the zero column
// part_w + c at that class's remaining steps below D_p, and from D_p on
// (steps the kernel skips after group ceil(D_p / 4) of the quarter warp)
// the zero column of its own class f.
__global__ void __launch_bounds__(BUILD_WARPS * 32)
k_sets_fill(const unsigned short *__restrict__ ent16, const long long *__restrict__ row_off16,
            int p_zero, int n_parts, int part_w, const int *__restrict__ counts,
            const int *__restrict__ set_frames, long long n_sets,
            const long long *__restrict__ goff, unsigned short *__restrict__ out,
            int *__restrict__ err) {
    __shared__ unsigned perm[BUILD_WARPS][4][SETS_MAX_PERMS];
    __shared__ int mult[BUILD_WARPS][4][SETS_MAX_PERMS];
    __shared__ int start[BUILD_WARPS][4][SETS_MAX_PERMS];
    __shared__ int n_perm[BUILD_WARPS][4];
    __shared__ int n_step[BUILD_WARPS][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int p = lane >> 3, f = lane & 7;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = warp; i < n_sets * n_parts; i += nwarp) {
        const int h = (int)(i / n_sets);
        const long long s = i - (long long)h * n_sets;
        const long long g0 = goff[i];
        const int steps = (int)(goff[i + 1] - g0) * 4;
        if (f == 0) {
            int m[8][8];
            int rows[8], cols[8];
            for (int c = 0; c < 8; ++c) cols[c] = 0;
            for (int ff = 0; ff < 8; ++ff) {
                const int d = set_frames[s * 32 + 8 * p + ff];
                rows[ff] = 0;
                for (int c = 0; c < 8; ++c) {
                    m[ff][c] = d >= 0 ? counts[(long long)d * 32 + h * 8 + c] : 0;
                    rows[ff] += m[ff][c];
                    cols[c] += m[ff][c];
                }
            }
            // this quarter warp's step count (Koenig: the fewest possible)
            int dq = 0;
            for (int k = 0; k < 8; ++k) dq = max(dq, max(rows[k], cols[k]));
            bool ok = dq <= steps;
            // pad to a regular matrix: every row and column sums to dq
            for (int ff = 0; ff < 8 && ok; ++ff)
                for (int c = 0; c < 8; ++c) {
                    const int t = min(dq - rows[ff], dq - cols[c]);
                    m[ff][c] += t;
                    rows[ff] += t;
                    cols[c] += t;
                }
            int np = 0, done = 0;
            while (ok && done < dq) {
                int col_of[8];
                if (np == SETS_MAX_PERMS || !perfect_matching(m, col_of)) {
                    ok = false;
                    break;
                }
                int mm = 0x7fffffff;
                unsigned packed = 0;
                for (int ff = 0; ff < 8; ++ff) {
                    mm = min(mm, m[ff][col_of[ff]]);
                    packed |= (unsigned)col_of[ff] << (4 * ff);
                }
                for (int ff = 0; ff < 8; ++ff) m[ff][col_of[ff]] -= mm;
                perm[w][p][np] = packed;
                mult[w][p][np] = mm;
                start[w][p][np] = done;
                done += mm;
                ++np;
            }
            if (!ok) {
                rspi_flag(err, RSPI_ERR_CAPACITY);
                np = 0;
                done = 0;
            }
            n_perm[w][p] = np;
            n_step[w][p] = done;
        }
        __syncwarp();
        const int np = n_perm[w][p];
        const int dq = n_step[w][p];
        const int d = set_frames[s * 32 + lane];
        // per class: current permutation index and offset within its run
        int ic[8], oc[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            ic[c] = 0;
            oc[c] = 0;
        }
        auto next_step = [&](int c) -> int {
            for (int guard = 0; guard <= SETS_MAX_PERMS && ic[c] < np; ++guard) {
                const int k = ic[c];
                if ((int)((perm[w][p][k] >> (4 * f)) & 15u) == c && oc[c] < mult[w][p][k])
                    return start[w][p][k] + oc[c]++;
                ++ic[c];
                oc[c] = 0;
            }
            return -1;
        };
        auto put = [&](int step, unsigned v) {
            out[((g0 + step / 4) * 32 + lane) * 4 + (step & 3)] = (unsigned short)v;
        };
        if (d >= 0 && np > 0) {
            const long long r0 = row_off16[d], r1 = row_off16[d + 1];
            for (long long rr = r0; rr < r1; ++rr) {
                for (int l2 = 0; l2 < 32; ++l2) {
                    const unsigned e = entry16_at(ent16, rr, l2);
                    if (e >= (unsigned)p_zero || (int)(e / (unsigned)part_w) != h) continue;
                    const unsigned loc = e - (unsigned)(h * part_w);
                    const int st = next_step((int)(loc & 7u));
                    if (st < 0) {
                        rspi_flag(err, RSPI_ERR_CAPACITY);
                        continue;
                    }
                    put(st, loc);
                }
            }
        }
        for (int c = 0; c < 8 && np > 0; ++c)
            for (int st = next_step(c); st >= 0; st = next_step(c))
                put(st, (unsigned)(part_w + c));
        for (int st = dq; st < steps; ++st) put(st, (unsigned)(part_w + f));
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// the screening kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint2 ld_entries(const uint2 *p, unsigned long long pol) {
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float4 ld_f4_hint(const float4 *p, unsigned long long pol) {
    float4 v;
    asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol)
                 : "memory");
    return v;
}

__device__ __forceinline__ void st_f4_hint(float4 *p, float4 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}

__device__ __forceinline__ void st_f32_hint(float *p, float v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
                 : "memory");
}

// Order-preserving key of (value, row) for a first-index argmax by an
// unsigned maximum: larger values give larger keys, NaN the largest (NumPy:
// the first NaN wins), -0 counts as +0; ties go to the smaller row.
__device__ __forceinline__ unsigned long long argmax_key(float v, unsigned row) {
    unsigned b = __float_as_uint(v + 0.f);
    b = isnan(v) ? 0xffffffffu : ((b & 0x80000000u) ? ~b : (b | 0x80000000u));
    return ((unsigned long long)b << 32) | (unsigned long long)(0xffffffffu - row);
}

__device__ __forceinline__ float4 f4_add(float4 a, float4 b) {
    const float2 lo = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
    const float2 hi = __fadd2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
    return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// The four photons of one group of a lane, summed as a tree of depth two:
// (v0 + v1) + (v2 + v3), four rows each.
__device__ __forceinline__ float4 group_sum(const unsigned char *tile, uint2 e) {
    const float4 v0 = *reinterpret_cast<const float4 *>(tile + ((e.x & 0xffffu) << 4));
    const float4 v1 = *reinterpret_cast<const float4 *>(tile + ((e.x >> 16) << 4));
    const float4 v2 = *reinterpret_cast<const float4 *>(tile + ((e.y & 0xffffu) << 4));
    const float4 v3 = *reinterpret_cast<const float4 *>(tile + ((e.y >> 16) << 4));
    return f4_add(f4_add(v0, v1), f4_add(v2, v3));
}

// Tensor memory (TMEM, 128 lanes x 512 columns of 32 bits per SM) as the
// store of the running part sums: warp w reaches lanes 32 (w % 4) .. + 31, so
// set s lives in lane quarter s % 4, columns 4 (s / 4) .. + 3 (one float4 per
// lane), for the first TMEM_SETS sets; later sets use the global scratch.
constexpr int TMEM_COLS = 512;
constexpr int TMEM_SETS = 4 * (TMEM_COLS / 4);

__device__ __forceinline__ void tmem_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_store4(unsigned taddr, float4 v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
                 "r"(__float_as_uint(v.x)), "r"(__float_as_uint(v.y)), "r"(__float_as_uint(v.z)),
                 "r"(__float_as_uint(v.w))
                 : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float4 tmem_load4(unsigned taddr) {
    unsigned x, y, z, w;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(x), "=r"(y), "=r"(z), "=r"(w)
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return make_float4(__uint_as_float(x), __uint_as_float(y), __uint_as_float(z),
                       __uint_as_float(w));
}

// Lane l of a set sums frame set_frames[32 s + l] over the set's groups of
// the part: groups alternate between two accumulators, then a0 + a1.  Each
// photon's value passes through at most ceil(G / 2) + 3 FP32 roundings in a
// part (G = the set's group count there).  With several parts, the parts
// before the last keep the running FP32 sum of (row, column 32 s + l) in
// tensor memory (sets below TMEM_SETS; the others in
// part_sums[cta][32 (s - TMEM_SETS) + l]); sets are then handed out by four
// queues, queue q = s % 4 to the warps w with w % 4 = q, so that a set meets
// its lane quarter in every part.  The last part adds the parts in FP64
// before the final rounding, stores the four rows' likelihoods in column
// 32 s + l and folds them into the column's argmax key (frame_max).
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
k_screen_sets(const float4 *__restrict__ lsl4, int num_rot, const double *__restrict__ init,
              const double *__restrict__ scales, const uint2 *__restrict__ groups,
              const long long *__restrict__ goff, const int *__restrict__ qgroups,
              const int *__restrict__ set_frames, int n_sets, int n_parts, int part_w,
              long long row_begin, long long row_end, float *__restrict__ ll,
              long long ll_stride, float4 *part_sums, unsigned long long *__restrict__ frame_max,
              int *err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ int next_set[4];
    __shared__ int abort_flag;
    __shared__ unsigned tmem_slot;
    float4 *tile = reinterpret_cast<float4 *>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned bytes = (unsigned)part_w * 16u;
    const unsigned mbar_a = smem_u32(&mbar), tile_a = smem_u32(tile);
    const unsigned long long keep = policy_evict_last(), stream_out = policy_evict_first();
    const bool split = n_parts > 1;   // running part sums (TMEM + scratch)
    if (threadIdx.x < 8) tile[part_w + threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    if (split && warp == 0) {
        // the whole tensor memory of the SM (one CTA per SM: 200 KB of
        // shared memory each); freed by the same warp at the end
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const unsigned tbase = split ? tmem_slot + ((unsigned)((warp & 3) * 32) << 16) : 0u;
    const int queue = split ? (warp & 3) : 0, n_queues = split ? 4 : 1;
    const int n_extra = n_sets > TMEM_SETS ? n_sets - TMEM_SETS : 0;
    float4 *ps = split ? part_sums + (long long)blockIdx.x * n_extra * 32 : nullptr;
    unsigned phase = 0;
    bool aborted = false;
    const long long n_tiles = (row_end - row_begin + 3) / 4;
    for (long long t = blockIdx.x; t < n_tiles && !aborted; t += gridDim.x) {
        const long long first = row_begin + 4 * t;
        const int nt = (int)min(4LL, row_end - first);
        for (int h = 0; h < n_parts; ++h) {
            tmem_fence_before();
            __syncthreads();   // every warp is done with the previous part
            tmem_fence_after();
            if (threadIdx.x == 0) {
                next_set[0] = next_set[1] = next_set[2] = next_set[3] = 0;
                const float4 *src = lsl4 + (t * n_parts + h) * (long long)part_w;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_a),
                             "r"(bytes)
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
                    " [%0], [%1], %2, [%3], %4;" ::"r"(tile_a),
                    "l"(src), "r"(bytes), "r"(mbar_a), "l"(stream_out)
                    : "memory");
                // the next part's slices into L2 while this one is gathered
                const long long nh = h + 1 < n_parts ? t * n_parts + h + 1
                                                     : (t + gridDim.x) * n_parts;
                if (t + (h + 1 < n_parts ? 0 : gridDim.x) < n_tiles) {
                    const char *nsrc = reinterpret_cast<const char *>(lsl4 + nh * part_w);
                    for (unsigned o = 0; o < bytes; o += 32768u)
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nsrc + o),
                                     "r"(min(32768u, bytes - o))
                                     : "memory");
                }
                // bounded wait for the copy
                const unsigned long long t0 = global_ns();
                unsigned ready = 0;
                while (!ready) {
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.u32 %0, 1, 0, p;\n\t}"
                        : "=r"(ready)
                        : "r"(mbar_a), "r"(phase)
                        : "memory");
                    if (!ready && global_ns() - t0 > (unsigned long long)WAIT_NS) break;
                }
                if (!ready) abort_flag = 1;
            }
            phase ^= 1u;
            __syncthreads();   // the part is in shared memory (or the wait ran out)
            if (abort_flag) {
                if (threadIdx.x == 0) {
                    rspi_flag(err, RSPI_ERR_TIMEOUT);
                    // wait (bounded) for the copy still in flight before leaving
                    const unsigned long long t0 = global_ns();
                    unsigned ready = 0;
                    while (!ready && global_ns() - t0 < (unsigned long long)WAIT_NS)
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                            "selp.u32 %0, 1, 0, p;\n\t}"
                            : "=r"(ready)
                            : "r"(mbar_a), "r"(phase ^ 1u)
                            : "memory");
                }
                aborted = true;
                break;
            }
            const bool last = h == n_parts - 1;
            double ini[4] = {0., 0., 0., 0.};
            if (last) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (k < nt) ini[k] = init[(first + k) / num_rot];
            }
            while (true) {
                int s = 0;
                if (lane == 0) s = queue + n_queues * atomicAdd(&next_set[queue], 1);
                s = __shfl_sync(RSPI_FULL_MASK, s, 0);
                if (s >= n_sets) break;
                const long long gi = (long long)h * n_sets + s;
                const long long g0 = goff[gi], g1 = goff[gi + 1];
                // the set runs ng groups; this lane's quarter warp stops after
                // its own nq (<= ng): its later gathers are not issued, so
                // they take no shared-memory wavefront
                const int ng = (int)(g1 - g0);
                const int nq = qgroups ? qgroups[gi * 4 + (lane >> 3)] : ng;
                float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
                const uint2 *gp = groups + g0 * 32 + lane;
                int k = 0;
                uint2 c0 = 0 < nq ? ld_entries(gp, keep) : make_uint2(0, 0);
                uint2 c1 = 1 < nq ? ld_entries(gp + 32, keep) : make_uint2(0, 0);
                for (; k + 1 < ng; k += 2, gp += 64) {
                    const uint2 n0 = k + 2 < nq ? ld_entries(gp + 64, keep) : make_uint2(0, 0);
                    const uint2 n1 = k + 3 < nq ? ld_entries(gp + 96, keep) : make_uint2(0, 0);
                    if (k < nq) a0 = f4_add(a0, group_sum(smem_raw, c0));
                    if (k + 1 < nq) a1 = f4_add(a1, group_sum(smem_raw, c1));
                    c0 = n0;
                    c1 = n1;
                }
                if (k < nq) a0 = f4_add(a0, group_sum(smem_raw, c0));
                const float4 sum = f4_add(a0, a1);
                const int col = s * 32 + lane;
                // this set's running sum: TMEM columns 4 (s / 4) of the lane
                // quarter, or the scratch
                const bool in_tmem = s < TMEM_SETS;
                const unsigned taddr = tbase + (unsigned)(4 * (s >> 2));
                float4 *pp = in_tmem ? nullptr : ps + (long long)(s - TMEM_SETS) * 32 + lane;
                if (!last) {
                    float4 run = sum;
                    if (h > 0) {
                        const float4 pv = in_tmem ? tmem_load4(taddr) : ld_f4_hint(pp, keep);
                        run = make_float4((float)((double)pv.x + (double)sum.x),
                                          (float)((double)pv.y + (double)sum.y),
                                          (float)((double)pv.z + (double)sum.z),
                                          (float)((double)pv.w + (double)sum.w));
                    }
                    if (in_tmem)
                        tmem_store4(taddr, run);
                    else
                        st_f4_hint(pp, run, keep);
                    continue;
                }
                float4 pv = make_float4(0.f, 0.f, 0.f, 0.f);
                if (h > 0) pv = in_tmem ? tmem_load4(taddr) : ld_f4_hint(pp, stream_out);
                const int d = set_frames[col];
                if (d < 0) continue;
                const double sc = scales[d];
                const float pr[4] = {pv.x, pv.y, pv.z, pv.w};
                const float sm[4] = {sum.x, sum.y, sum.z, sum.w};
                unsigned long long key = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k < nt) {
                        const float v = (float)(ini[k] * sc + ((double)pr[k] + (double)sm[k]));
                        st_f32_hint(ll + (first + k - row_begin) * ll_stride + col, v, stream_out);
                        const unsigned long long kk = argmax_key(v, (unsigned)(first + k));
                        key = kk > key ? kk : key;
                    }
                }
                atomicMax(frame_max + col, key);
            }
        }
    }
    // every warp is done with tensor memory; the allocating warp frees it
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    if (split && warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_slot),
                     "r"(TMEM_COLS)
                     : "memory");
}

// bad += entries that are not a staged column (< part_w + 8).
__global__ void k_sets_check(const unsigned short *__restrict__ e, long long n, int part_w,
                             int *__restrict__ bad) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    int cnt = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        cnt += (unsigned)e[i] >= (unsigned)(part_w + 8);
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(bad, cnt);
}

// Per column: the screened maximum and first-index argmax row of its frame
// from the key, into frame order; the key is reset for the next pass.
__global__ void k_frame_max_finalize(unsigned long long *__restrict__ frame_max,
                                     const int *__restrict__ frame_of_col, long long n_cols,
                                     double *__restrict__ max32, int *__restrict__ rmax32) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n_cols;
         k += stride) {
        const unsigned long long key = frame_max[k];
        frame_max[k] = 0ull;
        const int d = frame_of_col[k];
        if (d < 0) continue;
        const unsigned hi = (unsigned)(key >> 32);
        float v;
        if (hi == 0xffffffffu) {
            v = __uint_as_float(0x7fc00000u);   // NaN
        } else {
            const unsigned b = (hi & 0x80000000u) ? (hi & 0x7fffffffu) : ~hi;
            v = __uint_as_float(b);
        }
        max32[d] = (double)v;
        rmax32[d] = key == 0ull ? 0 : (int)(0xffffffffu - (unsigned)(key & 0xffffffffull));
    }
}

}  // namespace

extern "C" int rspi_sets_counts(const unsigned short *entries16, const long long *row_off16,
                                long long n_data, int p_zero, int n_parts, int part_w,
                                int *counts, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !counts || n_data <= 0 || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536 || n_parts < 1 || n_parts > SETS_MAX_PARTS || part_w < 8 ||
        part_w % 8 || (long long)n_parts * part_w < p_zero)
        return RSPI_ERR_ARG;
    k_sets_counts<<<rspi_blocks(n_data * 32, BUILD_WARPS * 32), BUILD_WARPS * 32, 0, stream>>>(
        entries16, row_off16, n_data, p_zero, n_parts, part_w, counts);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sets_group(const int *counts, const int *order, long long n, int n_parts,
                               int sweeps, int *set_frames, int *err, cudaStream_t stream) {
    if (!counts || !order || !set_frames || !err || n <= 0 || n > 0x7fffffffLL ||
        n_parts < 1 || n_parts > SETS_MAX_PARTS || sweeps < 0)
        return RSPI_ERR_ARG;
    const long long windows = (n + GROUP_W - 1) / GROUP_W;
    k_sets_group<<<(unsigned)windows, GROUP_W, 0, stream>>>(counts, order, n, n_parts, sweeps,
                                                           set_frames, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sets_steps(const int *counts, const int *set_frames, long long n_sets,
                               int n_parts, int *groups, int *quarter_groups,
                               cudaStream_t stream) {
    if (!counts || !set_frames || !groups || n_sets <= 0 || n_sets > 0x3ffffffLL ||
        n_parts < 1 || n_parts > SETS_MAX_PARTS)
        return RSPI_ERR_ARG;
    k_sets_steps<<<rspi_blocks(n_sets * n_parts, 256), 256, 0, stream>>>(
        counts, set_frames, n_sets, n_parts, groups, quarter_groups);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sets_fill(const unsigned short *entries16, const long long *row_off16,
                              int p_zero, int n_parts, int part_w, const int *counts,
                              const int *set_frames, long long n_sets, const long long *group_off,
                              unsigned short *entries, int *err, cudaStream_t stream) {
    if (!entries16 || !row_off16 || !counts || !set_frames || !group_off || !entries ||
        n_sets <= 0 || n_sets > 0x3ffffffLL || p_zero < 0 || p_zero % 32 ||
        p_zero + 32 > 65536 || n_parts < 1 || n_parts > SETS_MAX_PARTS || part_w < 8 ||
        part_w % 8 || part_w + 8 > 0xffff || (long long)n_parts * part_w < p_zero ||
        (reinterpret_cast<uintptr_t>(entries) & 7) != 0)
        return RSPI_ERR_ARG;
    k_sets_fill<<<rspi_blocks(n_sets * n_parts * 32, BUILD_WARPS * 32), BUILD_WARPS * 32, 0,
                  stream>>>(entries16, row_off16, p_zero, n_parts, part_w, counts, set_frames,
                            n_sets, group_off, entries, err);
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_sets_entries_check(const unsigned short *entries, long long n, int part_w,
                                       int *bad, cudaStream_t stream) {
    if (!entries || !bad || n <= 0 || part_w < 8 || part_w + 8 > 0xffff) return RSPI_ERR_ARG;
    k_sets_check<<<rspi_blocks(n, 256), 256, 0, stream>>>(entries, n, part_w, bad);
    RSPI_RETURN_LAUNCH();
}

extern "C" long long rspi_sets_part_sums_floats(long long n_sets, int n_ctas) {
    if (n_sets <= 0 || n_ctas <= 0) return -1;
    // the sets beyond the tensor-memory store (at least one set's room)
    const long long extra = n_sets > TMEM_SETS ? n_sets - TMEM_SETS : 1;
    return (long long)n_ctas * extra * 32 * 4;
}

extern "C" int rspi_screen_loglike_sets(const float *lslices_sets, long long num_rot,
                                        const double *init, const double *scales,
                                        const unsigned short *entries, const long long *group_off,
                                        const int *quarter_groups, const int *set_frames,
                                        long long n_sets, int n_parts,
                                        int part_w, long long row_begin, long long row_end,
                                        float *ll, long long ll_stride, float *part_sums,
                                        int part_sums_ctas, unsigned long long *frame_max,
                                        int warps_per_cta, int n_ctas, int *err,
                                        cudaStream_t stream) {
    if (!lslices_sets || !init || !scales || !entries || !group_off || !set_frames || !ll ||
        !frame_max || !err || n_sets <= 0 || n_sets > 0x3ffffffLL || num_rot <= 0 ||
        num_rot > 0x7fffffffLL || row_begin < 0 || row_end < row_begin ||
        row_end > 0x7fffffffLL || n_parts < 1 || n_parts > SETS_MAX_PARTS || part_w < 8 ||
        part_w % 8 || ll_stride < n_sets * 32 || warps_per_cta < 1 || warps_per_cta > 32)
        return RSPI_ERR_ARG;
    // several parts: the part sums' four lane quarters of tensor memory need
    // a warp in each quarter
    if (n_parts > 1 && (!part_sums || part_sums_ctas < 1 || warps_per_cta < 4))
        return RSPI_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(lslices_sets) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(entries) & 7) != 0 ||
        (reinterpret_cast<uintptr_t>(part_sums) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(frame_max) & 7) != 0)
        return RSPI_ERR_ARG;
    if (row_end == row_begin) return RSPI_OK;
    const size_t smem = (size_t)(part_w + 8) * sizeof(float4);
    if (smem > (size_t)SMEM_LIMIT - 1024) return RSPI_ERR_ARG;
    const long long n_tiles = (row_end - row_begin + 3) / 4;
    if (n_ctas <= 0) n_ctas = rspi_sm_count();
    if (n_parts > 1 && n_ctas > part_sums_ctas) n_ctas = part_sums_ctas;
    if (n_ctas > n_tiles) n_ctas = (int)n_tiles;
    float4 *ps = n_parts > 1 ? reinterpret_cast<float4 *>(part_sums) : nullptr;
    const float4 *src = reinterpret_cast<const float4 *>(lslices_sets);
    const uint2 *ent = reinterpret_cast<const uint2 *>(entries);
    if (warps_per_cta <= 16) {
        static RspiSmemOptIn optin;
        if (!rspi_smem_optin((const void *)k_screen_sets<512>, smem, optin)) return RSPI_ERR_CUDA;
        k_screen_sets<512><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            src, (int)num_rot, init, scales, ent, group_off, quarter_groups, set_frames,
            (int)n_sets, n_parts, part_w, row_begin, row_end, ll, ll_stride, ps, frame_max, err);
    } else {
        static RspiSmemOptIn optin;
        if (!rspi_smem_optin((const void *)k_screen_sets<1024>, smem, optin))
            return RSPI_ERR_CUDA;
        k_screen_sets<1024><<<n_ctas, warps_per_cta * 32, smem, stream>>>(
            src, (int)num_rot, init, scales, ent, group_off, quarter_groups, set_frames,
            (int)n_sets, n_parts, part_w, row_begin, row_end, ll, ll_stride, ps, frame_max, err);
    }
    RSPI_RETURN_LAUNCH();
}

extern "C" int rspi_frame_max_finalize(unsigned long long *frame_max, const int *frame_of_col,
                                       long long n_cols, double *max32, int *rmax32,
                                       cudaStream_t stream) {
    if (!frame_max || !frame_of_col || !max32 || !rmax32 || n_cols <= 0) return RSPI_ERR_ARG;
    k_frame_max_finalize<<<rspi_blocks(n_cols, 256), 256, 0, stream>>>(frame_max, frame_of_col,
                                                                       n_cols, max32, rmax32);
    RSPI_RETURN_LAUNCH();
}
