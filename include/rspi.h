/*
 * rspi.h -- C ABI of the B200 (sm_100a) RefSPI-MaxLP reconstruction hot path.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t,
 * launches asynchronously on that stream, allocates nothing and never
 * synchronises the host, so a whole iteration can be captured in a CUDA
 * graph.  The caller owns every buffer.  Returns RSPI_OK (0) or a negative
 * RSPI_ERR_* code for a bad argument or a failed launch; problems found on
 * the device (an out-of-range pixel index in the input, a bounded wait that
 * ran out) are written to the caller's `err` word (first error wins) and read
 * by the caller after the stream is synchronised.
 *
 * The reference (RefSPI-MaxLP) has no C ABI: its kernels are CuPy RawModule
 * launches driven from Python.  Each entry point below names the reference
 * code it replaces (file:line, relative to the reference project root).
 *
 * Layouts (row-major, pixel t = x*size + y, kernels.cu:13):
 *   state s0 = (isx*nsy + isy)*nd + idia (emc.py:71-77); likelihood row
 *   r = s0*num_rot + j for rotation angle j*pi/num_rot (emc.py:192,199).
 *   "sel" pixels: probmask == 0 (emc.py:95-98, kernels.cu:129), compacted in
 *   pixel order; a slice row holds p_pad >= n_sel values (p_pad % 32 == 0).
 */
#ifndef RSPI_H
#define RSPI_H

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSPI_OK 0
#define RSPI_ERR_ARG (-1)      /* bad size, pointer or option */
#define RSPI_ERR_INDEX (-2)    /* pixel / state index out of range in the input */
#define RSPI_ERR_CUDA (-3)     /* launch failed */
#define RSPI_ERR_TIMEOUT (-4)  /* a bounded device-side wait ran out */
#define RSPI_ERR_CAPACITY (-5) /* a value does not fit the packed layout */
#define RSPI_ERR_TOO_LARGE (-6) /* larger than the fixed scratch of a no-allocation entry
                                 * point (rspi_screen_candidates_noalloc only) */

/* Library version and build target, e.g. "rspi 0.1 sm_100a". */
const char *rspi_version(void);

/* Human-readable text for a status code. */
const char *rspi_status_string(int status);

/* ---------------------------------------------------------------- a1, a2
 * Photon-list setup.  Replaces dset.py:32-33,41-42 (ones_accum/multi_accum:
 * int64 exclusive prefix sums), dset.py:46-53 (mean_count, counts),
 * emc.py:129-132 (scales) and dset.py:74-83 (powder).  Bit-exact.
 *   totals[0] = sum(ones), totals[1] = sum(multi), totals[2] = sum(count_multi)
 *   mean_count = (totals[0] + totals[2]) / n_data;
 *   scales[d] = counts[d] / mean_count if need_scaling else 1.
 */
int rspi_photon_offsets(const int *ones, const int *multi, const int *count_multi,
                        long long n_data, long long *ones_accum, long long *multi_accum,
                        long long *counts, long long *totals, double *mean_count,
                        double *scales, int need_scaling, int *err, cudaStream_t stream);

/* powder[p] = (photons at p summed over frames) / n_data (dset.py:74-83).
 * Pixel indices outside [0, num_pix) set RSPI_ERR_INDEX in err and are skipped. */
int rspi_powder(const int *place_ones, long long n_ones, const int *place_multi,
                const int *count_multi, long long n_multi, long long num_pix,
                long long n_data, double *powder, int *err, cudaStream_t stream);

/* Likelihood entry lists (the layout calc_prob_all walks, kernels.cu:127-136,
 * restricted to probmask < 1).  Each frame's in-mask photons (ones with count
 * 1, multi with their counts) become 32-bit entries (sel_index << 16 | count)
 * packed into rows of 32 so that lane b holds sel_index % 32 == b: one warp
 * gather per row touches 32 distinct shared-memory banks.  Unused slots are
 * (b << 16 | 0).
 * Pass 1 writes frame_rows[d]; the caller forms row_off = exclusive scan
 * (rspi_scan_rows) and pass 2 fills entries[(row_off[d] + r)*32 + b].
 * Requires n_sel <= 65536 and every count <= 65535 (else RSPI_ERR_CAPACITY). */
int rspi_ll_entry_rows(const int *ones, const int *multi, const long long *ones_accum,
                       const long long *multi_accum, const int *place_ones,
                       const int *place_multi, const int *count_multi,
                       const int *pix2sel, long long num_pix, long long n_data,
                       int *frame_rows, long long *frame_sel_photons, int *err,
                       cudaStream_t stream);
int rspi_scan_rows(const int *frame_rows, long long n_data, long long *row_off,
                   cudaStream_t stream);
int rspi_ll_entry_fill(const int *ones, const int *multi, const long long *ones_accum,
                       const long long *multi_accum, const int *place_ones,
                       const int *place_multi, const int *count_multi,
                       const int *pix2sel, long long num_pix, long long n_data,
                       const long long *row_off, unsigned int *entries, int *err,
                       cudaStream_t stream);

/* ------------------------------------------------------------------- a4, a5
 * Holographic slices of every (shift, diameter) state, replacing
 * slice_gen_holo (kernels.cu:44-82, log_flag=0, rel_scale=scale=1) as
 * launched at emc.py:174-176 and 186-188:
 *   W[s0][p] = |model[p] + ff(pi*r*dia/size) * exp(i*phase)|^2 + bg[p]
 * and the masked sums msum[s0] = sum_{probmask<1} W[s0] (emc.py:177). */
int rspi_holo_slices(const double *model /* complex128, P */, const double *shiftx,
                     const double *shifty, const double *sphere_dia, long long n_states0,
                     long long size, const double *bg, const int *sel_pix, long long n_sel,
                     double *holo /* n_states0 x P */, double *msum, cudaStream_t stream);

/* EMC.sphere / EMC.ramp of one state (emc.py:244-254) over the P pixels, with
 * integer-centred x, y and r = sqrt(x^2 + y^2): sphere (nullable, doubles) =
 * (sin s - s cos s) / s^3, s = pi r dia / size (1e-5 where 0); ramp
 * (nullable, complex128) = e^{2 pi i (x sx + y sy) / size}. */
int rspi_sphere_ramp(long long size, double sx, double sy, double dia, double *sphere,
                     double *ramp, cudaStream_t stream);

/* vscale and per-state likelihood offsets (emc.py:181, 199):
 *   vscale = sum_sel powder / sum_s0 msum[s0] * n_states0,
 *   init[s0] = -(msum[s0] * vscale). */
int rspi_vscale_init(const double *msum, long long n_states0, const double *powder,
                     const int *sel_pix, long long n_sel, double *vscale, double *init,
                     cudaStream_t stream);

/* ------------------------------------------------------------------------ a6
 * Rotated log-slices restricted to sel pixels, replacing slice_gen with
 * log_flag=1 (kernels.cu:6-42) as launched at emc.py:191-193:
 *   L[s0*num_rot + j][c] = log(bilinear(W[s0])(R(j)(p-cen)+cen) + bg[p]),
 *   -1000 outside the detector or below 1e-20; p = sel_pix[c].
 * rot_cs[2*j], rot_cs[2*j+1] = cos, sin of angle j (host table).
 * out_dtype 0 = float32, 1 = float64, 2 = float16; rows are p_pad long, tail zeroed.
 * rows [row_begin, row_end) of the full S0*num_rot range are produced.
 * abs_max (nullable, float): raised to the largest |stored value| (the caller
 * zeroes it); it bounds the rounding error of the float32 form. */
int rspi_rot_log_slices(const double *holo, long long n_states0, long long num_rot,
                        const double *rot_cs, long long size, const double *bg,
                        const int *sel_pix, long long n_sel, long long p_pad,
                        long long row_begin, long long row_end, void *lslices,
                        int out_dtype, float *abs_max, cudaStream_t stream);

/* The same slices from a paired copy of the holographic slices:
 * rspi_holo_pairs writes holo_pairs[2 i], holo_pairs[2 i + 1] = holo[i],
 * holo[i + 1] (0 past the end; 16-byte aligned, 2 * n_states0 * size^2
 * doubles), so each row of a bilinear 2 x 2 neighbourhood is one 16-byte
 * load; rspi_rot_log_slices_pairs takes it in place of holo and gives
 * bit-identical output. */
int rspi_holo_pairs(const double *holo, long long n_states0, long long size,
                    double *holo_pairs, cudaStream_t stream);
int rspi_rot_log_slices_pairs(const double *holo_pairs, long long n_states0, long long num_rot,
                              const double *rot_cs, long long size, const double *bg,
                              const int *sel_pix, long long n_sel, long long p_pad,
                              long long row_begin, long long row_end, void *lslices,
                              int out_dtype, float *abs_max, cudaStream_t stream);

/* ------------------------------------------------------------------------ a7
 * Log-likelihood of frames x states, replacing calc_prob_all
 * (kernels.cu:116-137) launched once per (state, rotation) at emc.py:194-199:
 *   LL[r][d] = init[r / num_rot] * scales[d] + sum_entries count * L[r][sel]
 * One CTA owns `states_per_tile` consecutive rows, stages their slices in
 * shared memory and walks every frame's packed rows (a warp per frame,
 * frames taken in `frame_order`).  Accumulation is FP64.
 * slice_dtype / out_dtype: 0 = float32, 1 = float64.
 * Rows [row_begin, row_end) are computed: the slice of row r is read at
 * lslices + (r - row_begin) * p_pad and LL row r is written at
 * ll + (r - row_begin) * ll_stride. */
int rspi_loglike(const void *lslices, int slice_dtype, long long p_pad, long long num_rot,
                 const double *init, const double *scales, const unsigned int *entries,
                 const long long *row_off, const int *frame_order, long long n_data,
                 long long row_begin, long long row_end, void *ll, int out_dtype,
                 long long ll_stride, int states_per_tile, int warps_per_cta,
                 int n_ctas, cudaStream_t stream);

/* Streaming variant of rspi_loglike (form 1: 32-bit entries, FP64 slices and
 * output, bit-identical to rspi_loglike) and a plain screening kernel (form 0:
 * the 16-bit entries of rspi_ll16_entry_fill, two rows per 32-bit word, FP32
 * slices, FP32 sums and output: LL32[r][d] = float(init[r/num_rot]*scales[d]
 * + FP32 sum of the frame's FP32 slice values)).  Each warp owns a contiguous range
 * of frames holding an equal share of the entry words and streams it with a
 * prefetch across frame boundaries; frames are processed in index order
 * (no frame_order).  row_off are the entry-row offsets of that form. */
int rspi_loglike_stream(int form, const void *lslices, long long p_row, long long num_rot,
                        const double *init, const double *scales, const void *entries,
                        const long long *row_off, long long n_data, long long row_begin,
                        long long row_end, void *ll, long long ll_stride, int states_per_tile,
                        int warps_per_cta, int n_ctas, cudaStream_t stream);

/* Largest states_per_tile whose slices fit in shared memory (0 if none). */
int rspi_loglike_max_tile(long long p_pad, int slice_dtype);

/* ---------------------------------------------------------- a7 screened form
 * The chosen likelihood: an FP32 screening pass, candidate selection with a
 * rigorous error bound, and FP64 rescoring of the candidates (replaces the
 * same calc_prob_all launches as rspi_loglike, kernels.cu:116-137).
 *
 * rspi_ll16_entry_rows / _fill: 16-bit photon entries for the screening
 * pass.  Each in-mask photon is one entry holding its sel index (a pixel with
 * k photons gives k entries); lane b of a row holds an index = b mod 32.
 * frame_rows[d] is even; with row_off = rspi_scan_rows(frame_rows) the word
 * (pair q, lane b) at entries[q*64 + 2b .. 2b+1] holds rows 2q and 2q+1.
 * Unused slots hold p_zero + b, where the slice rows are zero
 * (p_zero = p_row - 32, p_zero >= n_sel, p_row <= 65536). */
int rspi_ll16_entry_rows(const int *ones, const int *multi, const long long *ones_accum,
                         const long long *multi_accum, const int *place_ones,
                         const int *place_multi, const int *count_multi, const int *pix2sel,
                         long long num_pix, long long n_data, int p_zero, int *frame_rows,
                         int *err, cudaStream_t stream);
int rspi_ll16_entry_fill(const int *ones, const int *multi, const long long *ones_accum,
                         const long long *multi_accum, const int *place_ones,
                         const int *place_multi, const int *count_multi, const int *pix2sel,
                         long long num_pix, long long n_data, int p_zero,
                         const long long *row_off, unsigned short *entries,
                         cudaStream_t stream);

/* Frame quads with four rows per tile: one 16-byte gather brings a photon's
 * value in all four rows.  The likelihood columns [0, p_zero) are cut into
 * n_parts (1-4) parts of part_w columns (part_w % 8 == 0, n_parts * part_w
 * >= p_zero), each staged with 8 zero columns after it.  Lane 8 u + j of a
 * group holds frame u's photons of part h whose local column (column -
 * h part_w) is = j (mod 8), as q = local / 8, four per group; the k-th
 * photon of (h, j) goes to group k / 4, slot k mod 4; other slots hold
 * q = part_w / 8.
 * rspi_quad4_entry_groups: groups[d * n_parts + h] = ceil(max_j n_hj / 4).
 * The caller forms quads (quad_slot[d] = 4 q + u, quad_frames), takes per
 * (quad, part) the largest count of its frames and scans them part-major
 * into group_off[n_parts * n_quads + 1] (range h * n_quads + q).
 * rspi_quad4_entry_fill: total_groups * 128 16-bit entries (8-byte aligned).
 * rspi_screen_loglike7: the likelihood rows from them.  With several parts
 * the running FP32 sum of each (CTA, row, frame slot) sits in part_sums
 * (rspi_quad4_part_sums_floats(n_quads, part_sums_ctas) floats; at most
 * part_sums_ctas CTAs run) and the parts' sums are added in FP64 before the
 * final FP32 rounding: within the FP32 error bound with each frame's
 * summation length max(entry rows, its quad's largest part group count). */
int rspi_quad4_entry_groups(const unsigned short *entries16, const long long *row_off16,
                            long long n_data, int p_zero, int n_parts, int part_w, int *groups,
                            cudaStream_t stream);
int rspi_quad4_entry_fill(const unsigned short *entries16, const long long *row_off16,
                          long long n_data, int p_zero, int n_parts, int part_w,
                          const int *quad_slot, const long long *group_off, long long n_quads,
                          long long total_groups, unsigned short *narrow, cudaStream_t stream);
long long rspi_quad4_part_sums_floats(long long n_quads, int n_ctas);
int rspi_screen_loglike7(const float *lslices, long long p_row, long long num_rot,
                         const double *init, const double *scales, const unsigned short *narrow,
                         const long long *group_off, const int *quad_frames, long long n_quads,
                         int n_parts, int part_w, long long row_begin, long long row_end,
                         float *ll, long long ll_stride, float *part_sums, int part_sums_ctas,
                         int warps_per_cta, int n_ctas, cudaStream_t stream);

/* Frame sets (the chosen screening kernel).  Frames are taken 32 at a time:
 * set s holds frames set_frames[32 s + l] (l = lane, -1 for none) and writes
 * them to likelihood column 32 s + l (the caller orders frames, e.g. by
 * photon count, so a set's frames need alike work; the likelihood matrix
 * then has n_sets * 32 columns in that order).  Lane 8 p + f of a set is
 * frame f of quarter warp p.  The likelihood columns [0, p_zero) are cut
 * into n_parts (1-4) parts of part_w columns (part_w % 8 == 0,
 * n_parts * part_w >= p_zero), each staged in shared memory as four FP32
 * rows per column with 8 zero columns after it.
 * rspi_sets_counts: counts[d * 32 + 8 h + c] = frame d's photons in part h of
 * local column class c (local column mod 8), from the 16-bit entries of
 * rspi_ll16_entry_fill (p_zero = their zero column).
 * rspi_sets_group: set_frames[32 * ceil(n_data / 32)] from `order` (the
 * frames by decreasing photon count, a permutation of [0, n_data)) and
 * rspi_sets_counts' counts: per window of 256 consecutive ranks, quarters of
 * eight frames built greedily (each from the longest frame left, adding the
 * frame that keeps sum over parts of max(largest frame, largest class total)
 * smallest), then up to `sweeps` sweeps over every pair of the window's
 * quarters making the best cost-lowering exchange of one frame each, then
 * the quarters in decreasing cost, four to a set (-1 for empty slots).
 * Deterministic (integer costs, ties to the lower index).  An `order` entry
 * outside [0, n_data) sets *err = RSPI_ERR_INDEX and is left out.  Replaces
 * the rank-interleaved order (frame of rank 32 s + p + 4 f in lane 8 p + f)
 * as the library's default.
 * rspi_sets_steps: quarter_groups[(h * n_sets + s) * 4 + p] (NULL: not
 * written) = ceil(D_p / 4), D_p the fewest steps quarter warp p of set s
 * needs in part h: max(largest frame count, largest class total over its
 * eight frames) (Koenig's edge-colouring bound); groups[h * n_sets + s] =
 * the largest of the four.  The caller scans the groups part-major into
 * group_off[n_parts*n_sets + 1].
 * rspi_sets_fill: group_off[last] * 128 16-bit entries (8-byte aligned,
 * prefilled by the caller with any value <= part_w + 7): entry
 * ((g * 32 + lane) * 4 + k) is the local column the lane reads at step
 * 4 (g - g0) + k of its (set, part) range [g0, g1).  A quarter warp runs
 * its own D_q steps (max of its largest frame count and largest class
 * total), in each of which its eight lanes read eight distinct classes (a
 * Birkhoff-von Neumann decomposition of the count matrix padded to a
 * regular one), real photons first, the zero column part_w + class
 * otherwise; from step D_q on each lane holds the zero column of its own
 * class (rspi_screen_loglike_sets skips those groups of the quarter warp
 * when given quarter_groups).  A schedule that cannot be built sets
 * *err = RSPI_ERR_CAPACITY. */
int rspi_sets_counts(const unsigned short *entries16, const long long *row_off16,
                     long long n_data, int p_zero, int n_parts, int part_w, int *counts,
                     cudaStream_t stream);
int rspi_sets_group(const int *counts, const int *order, long long n_data, int n_parts,
                    int sweeps, int *set_frames, int *err, cudaStream_t stream);
int rspi_sets_steps(const int *counts, const int *set_frames, long long n_sets, int n_parts,
                    int *groups, int *quarter_groups, cudaStream_t stream);
int rspi_sets_fill(const unsigned short *entries16, const long long *row_off16, int p_zero,
                   int n_parts, int part_w, const int *counts, const int *set_frames,
                   long long n_sets, const long long *group_off, unsigned short *entries,
                   int *err, cudaStream_t stream);

/* Rotated log-slices in the layout of rspi_screen_loglike_sets: rows taken
 * four at a time from row_begin, columns cut into parts:
 * out[(((r - row_begin) / 4 * n_parts + h) * part_w + c) * 4 + (r - row_begin) % 4]
 * is row r at column h * part_w + c (zero past n_sel); rows of a partial
 * last tile beyond row_end are not written.  holo_pairs as for
 * rspi_rot_log_slices_pairs; out 16-byte aligned.  holo_quads32 NULL: the
 * values of rspi_rot_log_slices rounded to FP32 (identical bits).
 * holo_quads32 given (rspi_holo_quads32: per pixel i of every state the four
 * bilinear corners W[i], W[i + 1], W[i + size], W[i + size + 1] in FP32,
 * 16-byte aligned, 4 * n_states0 * size^2 floats): the interpolation and
 * the log in FP32 (lg2.approx times ln 2), |L32 - L| <= 2^-24 (16 + 7 |L|),
 * with values at or below 2e-20 (and the in-detector test) in FP64 so the
 * -1000 sentinel falls where the reference's does; the caller's candidate
 * threshold must cover the extra error (rows + 23 with abs_max >= 1). */
int rspi_holo_quads32(const double *holo, long long n_states0, long long size,
                      float *holo_quads32, cudaStream_t stream);
int rspi_rot_log_slices_sets(const double *holo_pairs, const float *holo_quads32,
                             long long n_states0, long long num_rot, const double *rot_cs,
                             long long size, const double *bg, const int *sel_pix,
                             long long n_sel, int n_parts, int part_w, long long row_begin,
                             long long row_end, float *out, float *abs_max, cudaStream_t stream);

/* FP32 screening likelihood of rows [row_begin, row_end) from those slices
 * (one bulk copy per tile part into shared memory) and the set entries: lane l
 * of set s sums its frame's photons in the four rows (two alternating FP32
 * accumulators over the groups, each group's four photons as a depth-two
 * tree: at most ceil(G/2) + 3 roundings per value and part, G = the set's
 * groups in the part); the parts are added in FP64 before the final
 * rounding, the running sum of parts before the last kept in the SM's
 * tensor memory for the first 512 sets (each CTA allocates all 512 TMEM
 * columns and frees them before it ends; warps_per_cta >= 4) and in
 * part_sums for the others (rspi_sets_part_sums_floats(n_sets,
 * part_sums_ctas) floats, 16-byte aligned; at most part_sums_ctas CTAs
 * run).  With quarter_groups (rspi_sets_steps; NULL: every quarter warp
 * runs its set's groups) a quarter warp stops gathering after its own
 * groups.  LL32 of row r, frame set_frames[c] goes to
 * ll[(r - row_begin) * ll_stride + c] (ll_stride >= n_sets * 32), and
 * frame_max[c] (zero before the first launch of a pass) takes the unsigned
 * maximum of an order-preserving (value, row) key, read and reset by
 * rspi_frame_max_finalize.  A bulk copy that does not complete within 1 s
 * sets *err = RSPI_ERR_TIMEOUT and the kernel returns.  Requires every entry
 * <= part_w + 7 (check with rspi_sets_entries_check). */
long long rspi_sets_part_sums_floats(long long n_sets, int n_ctas);
/* *bad += the entries of entries[0, n) that are not a staged column
 * (< part_w + 8): the check of rspi_sets_fill's output before the first
 * launch. */
int rspi_sets_entries_check(const unsigned short *entries, long long n, int part_w, int *bad,
                            cudaStream_t stream);
int rspi_screen_loglike_sets(const float *lslices_sets, long long num_rot, const double *init,
                             const double *scales, const unsigned short *entries,
                             const long long *group_off, const int *quarter_groups,
                             const int *set_frames,
                             long long n_sets, int n_parts, int part_w, long long row_begin,
                             long long row_end, float *ll, long long ll_stride,
                             float *part_sums, int part_sums_ctas,
                             unsigned long long *frame_max, int warps_per_cta, int n_ctas,
                             int *err, cudaStream_t stream);

/* Per-frame screened maximum and first-index argmax (NumPy's rules: the
 * first NaN wins) from the keys of rspi_screen_loglike_sets: for every
 * column c with frame d = frame_of_col[c] >= 0, max32[d] and rmax32[d]; the
 * keys are reset to zero for the next pass (replaces rspi_frame_reduce's
 * pass over the FP32 matrix, emc.py:207-216). */
int rspi_frame_max_finalize(unsigned long long *frame_max, const int *frame_of_col,
                            long long n_cols, double *max32, int *rmax32, cudaStream_t stream);

/* *max_index = largest value in a 16-bit entry array. */
int rspi_entries16_check(const unsigned short *entries, long long n_entries,
                         unsigned *max_index, cudaStream_t stream);

/* Candidates: state r of frame d is kept when LL32[r][d] >= max32[d] - delta
 * - 2*eps_d or r == rmax32[d] (the screened first-index argmax, so a frame
 * whose values are all NaN keeps its first NaN row), eps_d = 2^-24 ((rows_d + 8) * photons_d * lmax + |max32| + delta + 1)
 * bounding |LL32 - LL64| (photons_d = in-mask photons, rows_d from row_off16,
 * lmax = largest |slice value|).  Writes cand_n[d], the exclusive offsets
 * cand_off (n_data + 1, total at [n_data]), the pairs (cand_d, cand_r) up to
 * `capacity` (beyond it RSPI_ERR_CAPACITY goes to err), the threshold thr[d]
 * and noncand[d] = sum over dropped states of exp(LL32 - max32[d]).
 * cnt_part is scratch of n_data * 32 ints. */
int rspi_screen_candidates(const float *ll, long long n_rows, long long n_data,
                           const double *max32, const int *rmax32, const long long *frame_photons,
                           const long long *row_off16, const float *lmax, double delta,
                           int *cnt_part, int *cand_n, double *noncand, double *thr,
                           long long *cand_off, long long capacity, int *cand_d, int *cand_r,
                           int *err, cudaStream_t stream);

/* rspi_screen_candidates without the cnt_part scratch argument, for callers
 * that cannot allocate device memory (no counterpart in the reference).  The
 * scratch is a fixed device array inside the library, sized for at most
 * 65536 frames (8 MiB per GPU, held until the process exits); more frames
 * return RSPI_ERR_TOO_LARGE.  The first call on a device looks the array up
 * (make it before any stream capture); calls that overlap on the GPU share
 * the array and race, so the caller serialises them.  Outputs are those of
 * rspi_screen_candidates. */
int rspi_screen_candidates_noalloc(const float *ll, long long n_rows, long long n_data,
                                   const double *max32, const int *rmax32,
                                   const long long *frame_photons, const long long *row_off16,
                                   const float *lmax, double delta, int *cand_n,
                                   double *noncand, double *thr, long long *cand_off,
                                   long long capacity, int *cand_d, int *cand_r, int *err,
                                   cudaStream_t stream);

/* rspi_screen_candidates over a likelihood matrix whose n_cols columns hold
 * frames in another order: column c holds frame frame_of_col[c] (-1: none);
 * the outputs are per frame as in rspi_screen_candidates.  With cand_slot
 * (n_data * 32 ints of scratch) the matrix is read once: the counting pass
 * records each thread's candidate rows when it has one or two, a compaction
 * writes those frames' lists, and only frames where one thread (rows
 * r = t mod 32) met three or more candidates are scanned again -- the same
 * lists in the same order as without it. */
int rspi_screen_candidates_cols(const float *ll, long long n_rows, long long n_cols,
                                const int *frame_of_col, long long n_data, const double *max32,
                                const int *rmax32, const long long *frame_photons,
                                const long long *row_off16, const float *lmax, double delta,
                                int *cnt_part, int *cand_n, double *noncand, double *thr,
                                long long *cand_off, long long capacity, int *cand_d,
                                int *cand_r, int *cand_slot, int *err, cudaStream_t stream);

/* FP64 rescoring of every candidate, in the summation order of rspi_loglike
 * (so the values equal the FP64 form's), written to cand_ll and into ll32;
 * then per frame the first-index argmax, maximum and
 * logz = max + log(sum_cand exp(LL64 - max) + noncand * exp(max32 - max)).
 * Candidates are regrouped by likelihood row (scratch row_cnt[n_rows],
 * row_cand_off[n_rows + 1], row_cand[capacity]); one CTA computes a row's
 * FP64 rotated slice (p_pad values, as rspi_rot_log_slices) in shared
 * memory and rescores that row's candidate frames.  A row too long for
 * shared memory (p_pad * 8 bytes above 220 KB) is built in row_scratch
 * instead (scratch_rows x p_pad doubles, one slot per CTA; required then,
 * ignored otherwise). */
int rspi_rescore(const int *cand_d, const int *cand_r, const long long *cand_off,
                 long long n_data, long long capacity, long long n_rows, const double *holo,
                 long long num_rot, const double *rot_cs, long long size, const double *bg,
                 const int *sel_pix, long long n_sel, long long p_pad, const double *init,
                 const double *scales, const unsigned int *entries32,
                 const long long *row_off32, int *row_cnt, long long *row_cand_off,
                 int *row_cand, double *cand_ll, float *ll32, const double *max32,
                 const double *noncand, double *maxll, int *rmax, double *logz,
                 double *row_scratch, long long scratch_rows, cudaStream_t stream);

/* rspi_rescore for a likelihood matrix with n_cols columns in which frame d
 * is column col_of_frame[d]. */
int rspi_rescore_cols(const int *cand_d, const int *cand_r, const long long *cand_off,
                      long long n_data, long long capacity, long long n_rows, const double *holo,
                      long long num_rot, const double *rot_cs, long long size, const double *bg,
                      const int *sel_pix, long long n_sel, long long p_pad, const double *init,
                      const double *scales, const unsigned int *entries32,
                      const long long *row_off32, int *row_cnt, long long *row_cand_off,
                      int *row_cand, double *cand_ll, float *ll32, long long n_cols,
                      const int *col_of_frame, const double *max32, const double *noncand,
                      double *maxll, int *rmax, double *logz, double *row_scratch,
                      long long scratch_rows, cudaStream_t stream);

/* ------------------------------------------------------------------- a8, a9
 * Per-frame reduction over all states of LL (n_rows x n_data, FP64 or FP32):
 * first-index max/argmax (emc.py:208-209) and the FP64 log-sum-exp
 * logz[d] = max + log(sum_r exp(LL[r][d] - max)) (standard EMC
 * normalisation; absent from the reference run path). */
int rspi_frame_reduce(const void *ll, int ll_dtype, long long n_rows, long long n_data,
                      double *maxll, int *rmax, double *logz, cudaStream_t stream);

/* ----------------------------------------------------------------------- a10
 * Posterior-weighted merge, composed from the reference's merge_all
 * (kernels.cu:139-152) and slice_merge (kernels.cu:84-114), which it ships
 * but never launches:
 *   num[s0](q) = sum_j R_j^T[sum_d P[s0*R+j][d] K_d](q),
 *   w[r] = sum_d P[r][d] scales[d], den[s0](q) = sum_j w[s0*R+j] C_j(q),
 *   intens = num / den (0 where den == 0), C_j = R_j^T 1,
 * with P = exp(LL - logz[d]) counted when P >= p_min.
 *
 * rspi_posterior_pairs: the (frame, row, LL) pairs with P >= p_min from a
 * full FP64 likelihood matrix (count / scan / fill as rspi_screen_candidates;
 * total at off[n_data]).  The screened form passes its candidate list instead.
 * rspi_merge_coverage: C (num_rot x P), once per geometry.
 * rspi_merge: zeroes num and w, scatters every pair's photons, finalises. */
int rspi_posterior_pairs(const double *ll, long long n_rows, long long n_data,
                         const double *logz, double p_min, int *cnt_part, int *cnt,
                         long long *off, long long capacity, int *pair_d, int *pair_r,
                         double *pair_ll, int *err, cudaStream_t stream);
int rspi_merge_coverage(long long num_rot, const double *rot_cs, long long size, double *cov,
                        cudaStream_t stream);
int rspi_merge(const int *pair_d, const int *pair_r, const double *pair_ll,
               const long long *pair_total, long long capacity, const double *logz,
               double p_min, const double *scales, const int *ones, const int *multi,
               const long long *ones_accum, const long long *multi_accum,
               const int *place_ones, const int *place_multi, const int *count_multi,
               long long n_states0, long long num_rot, const double *rot_cs, long long size,
               const double *cov, double *num, double *den, double *w, double *intens,
               cudaStream_t stream);

/* ----------------------------------------------------------------- a11-a14
 * MaxLP M-step (maxLP.py:304-340).  Frames carry a reference-state index
 * fstate[d] into ref_params (n_ref x 3: shiftx, shifty, diameter) and a
 * rotation index frot[d] into rot_cs (cos(-a), sin(-a)).
 *
 * rspi_maxlp_frame_params: from the E-step argmax rmax[d] (emc.py:218-224):
 *   fstate = rmax / num_rot, frot = rmax % num_rot, nstate[s] = #frames. */
int rspi_maxlp_frame_params(const int *rmax, long long n_data, long long num_rot,
                            long long n_ref, int *fstate, int *frot, int *nstate,
                            int *err, cudaStream_t stream);

/* Photon histogram of every phaser pixel over reference states:
 *   hist[m][s] = sum over frames d with fstate[d]==s of K_d(u_d(t_m)),
 * u_d(t) = rint(R(-ang_d) q_t * size + size//2) (maxLP.py:245-253), scattered
 * from each photon to the model pixels that map onto it.  The index
 * arithmetic is two products and a sum per coordinate without fused
 * multiply-add, so it is bit-exact with the FP64 restatement.
 * mask_idx[t] = m for phaser pixels (maxLP.py:88), -1 elsewhere.  hist must be
 * zeroed by the caller (n_mask x n_ref int32). */
int rspi_maxlp_histogram(const int *ones, const int *multi, const long long *ones_accum,
                         const long long *multi_accum, const int *place_ones,
                         const int *place_multi, const int *count_multi, long long n_data,
                         const int *fstate, const int *frot, const double *rot_cs,
                         long long size, const int *mask_idx, long long n_mask,
                         long long n_ref, int *hist, int *err, cudaStream_t stream);

/* The same histogram from a table built once per rotation table (what the
 * library's M-step uses).  rspi_maxlp_pixel_map lists, for each rotation j
 * of rot_cs and detector pixel p, the phaser rows m whose pixel maps onto p
 * (on an even detector a map onto column `size` of row x is listed under
 * pixel (x + 1, 0), as rspi_maxlp_histogram aliases it): rows
 * map_rows[map_off[j * size^2 + p] .. map_off[j * size^2 + p + 1]), in no
 * particular order.  Scratch cnt: num_rot * size^2 ints; map_off:
 * num_rot * size^2 + 1; map_rows: num_rot * n_mask (each pixel maps to one
 * detector pixel per rotation at most).  rspi_maxlp_histogram_map adds each
 * photon of frame d to the rows listed under its pixel for rotation
 * frot[d]: the same integer sums as rspi_maxlp_histogram (hist zeroed by
 * the caller; a rotation outside [0, num_rot) or a pixel outside the
 * detector sets *err = RSPI_ERR_INDEX). */
int rspi_maxlp_pixel_map(const double *rot_cs, long long num_rot, long long size,
                         const int *mask_idx, int *cnt, long long *map_off, int *map_rows,
                         cudaStream_t stream);
int rspi_maxlp_histogram_map(const int *ones, const int *multi, const long long *ones_accum,
                             const long long *multi_accum, const int *place_ones,
                             const int *place_multi, const int *count_multi, long long n_data,
                             const int *fstate, const int *frot, long long num_rot,
                             long long size, const long long *map_off, const int *map_rows,
                             long long n_ref, int *hist, int *err, cudaStream_t stream);

/* Pattern search of a set of model pixels (maxLP.py:154-197): for each pixel
 * t = pixels[i] (its histogram row hist_row[i]) run <= num_iter iterations over
 * the 33x33 candidate grid.  rescale_mode 0: per-candidate rescale
 * (ring pass, maxLP.py:186-187); 1: the scalar rescale of the mode (main pass).
 *
 * n_modes independent models are searched in one launch (n_modes = 1 is the
 * reference's single model; num_modes, parsed at emc.py:59, is otherwise
 * unused there).  Mode m owns model fconv[m*P .. (m+1)*P) (complex128,
 * updated in place), histogram columns m*n_ref .. (m+1)*n_ref of each
 * n_modes*n_ref-wide hist row, frame counts nstate[m*n_ref ..] and, in the
 * main pass, rescale[m].  The means over frames divide by the mode's frame
 * count sum_s nstate[m*n_ref + s] (N for one mode); a mode without frames
 * keeps its model.  With rescale_out != NULL the per-pixel rescale of the
 * final value (maxLP.py:328) goes to rescale_out[m*n_pix + i] (NaN for a
 * mode without frames). */
int rspi_maxlp_pattern(double *fconv, const int *pixels, const int *hist_row,
                       long long n_pix, const int *hist, long long n_ref,
                       const int *nstate, long long n_modes, const double *ref_params,
                       long long size, int rescale_mode, const double *rescale,
                       int num_iter, double *rescale_out, cudaStream_t stream);

/* rspi_maxlp_pattern with an FP32 screening pass per iteration: every
 * candidate is first evaluated in FP32 with a rigorous bound on its distance
 * from the FP64 value; only the candidates that can still be the argmax
 * (the finalists; every candidate without a finite bound) are evaluated in
 * FP64, with the same sums and roundings as rspi_maxlp_pattern, so the
 * chosen candidates, and fconv and rescale_out, are bit-identical to it.
 * Pixels with more than 1024 populated states, counts >= 2^24, or ring
 * pixels without photons run the FP64 iterations.  stats (device, 3
 * counters, NULL for none; the caller zeroes them) accumulates [iterations
 * through the screen, iterations of the FP64 pass, finalists]. */
int rspi_maxlp_pattern_screened(double *fconv, const int *pixels, const int *hist_row,
                                long long n_pix, const int *hist, long long n_ref,
                                const int *nstate, long long n_modes, const double *ref_params,
                                long long size, int rescale_mode, const double *rescale,
                                int num_iter, double *rescale_out, unsigned long long *stats,
                                cudaStream_t stream);

/* The error of the FP32 screen's log2 (lg2.approx.f32) over every float in
 * [lo, hi] (0 < lo <= hi): out[0] (device double) = the largest
 * |lg2(x) - log2(x)| / (2^-21 + 2^-22 |lg2(x)|), the bound the screened
 * pattern search uses (it needs out[0] <= 1 on [2^-100, 2^100]); out[1] =
 * the largest absolute error. */
int rspi_log2_error_max(float lo, float hi, double *out, cudaStream_t stream);

/* Per-pixel, per-frame phaser API (the reference's get_photons_pixel,
 * get_fref_d, get_rescale_pixel, get_logq_pixel; maxLP.py:181-253), without
 * the state aggregation of rspi_maxlp_pattern.
 *
 * rspi_maxlp_pixel_frames: for frame d = d_vals[i] (d = i when d_vals is
 * NULL), k_out[i] = photons of frame d at the flat detector column
 * rint(R q_t size) + size/2 of model pixel t (rot_cs[2d], rot_cs[2d+1] =
 * cos, sin of -angle_d; 0 off the matrix) and fref_out[2i], [2i+1] = the
 * complex reference amplitude ff(pi qrad dia) e^{2 pi i q . shift} of
 * fparams[3d..3d+2] = (shift x, shift y, diameter).  A d_vals entry outside
 * [0, n_data) sets RSPI_ERR_INDEX and gives 0.
 *
 * rspi_maxlp_pixel_values: for candidate c (complex cands[2c], [2c+1]) over
 * the n frames: mode 0 writes mean_d k_d / mean_d |f_c + fref_d|^2 (the
 * rescale); mode 1 writes mean_d k_d log(rho w) - mean_d rho w, w =
 * |f_c + fref_d|^2, rho = rescale_vec[c] if given, else rescale. */
int rspi_maxlp_pixel_frames(int t, long long size, const int *d_vals, long long n_vals,
                            const int *ones, const int *multi, const long long *ones_accum,
                            const long long *multi_accum, const int *place_ones,
                            const int *place_multi, const int *count_multi, long long n_data,
                            const double *rot_cs, const double *fparams, double *k_out,
                            double *fref_out, int *err, cudaStream_t stream);
int rspi_maxlp_pixel_values(const double *cands, long long n_c, const double *k,
                            const double *fref, long long n, int mode, double rescale,
                            const double *rescale_vec, double *out, cudaStream_t stream);

/* Sphere transform ff(pi qrad dia) of every model pixel into sphere (P
 * doubles, maxLP.py:266-269) and/or the holographic amplitude
 * fobj + ff e^{2 pi i (qx shift_x + qy shift_y)} into fcalc (P complex128,
 * maxLP.py:260-264). */
int rspi_maxlp_fcalc(long long size, double dia, double sx, double sy, const double *fobj,
                     double *sphere, double *fcalc, cudaStream_t stream);

/* Polar grid search of the per-pixel MaxLP negative log-likelihood (the
 * comparison for the L-BFGS update of rspi_nll; no reference counterpart):
 * for each pixel t = pixels[i] (histogram row hist_row[i], one mode),
 *   NLL_t(F) = sum_s S_s |F + r_s|^2 - sum_s K_t[s] log |F + r_s|^2,
 * S_s = sum of scales[d] over frames with fstate[d] == s (written to
 * ssum[n_ref]), over F = a_j e^{i phi_i}, phi_i = 2 pi i / n_phase,
 * a_j = A (j + 1) / n_amp, A = sqrt(sum_s K_t[s] / sum_s S_s) + max_s |r_s|.
 * The lowest value (first index on ties) becomes fconv[t]; best_nll[i] gets
 * it (without the F-independent sum_d k_dt log scale_d).  A pixel without
 * frames keeps its value (best_nll 0). */
int rspi_maxlp_grid(double *fconv, const int *pixels, const int *hist_row, long long n_pix,
                    const int *hist, long long n_ref, const int *fstate, const double *scales,
                    long long n_data, const double *ref_params, long long size, int n_phase,
                    int n_amp, double *ssum, double *best_nll, int *err, cudaStream_t stream);

/* Mean of n values into *out (the global rescale, maxLP.py:329). */
int rspi_mean(const double *vals, long long n, double *out, cudaStream_t stream);

/* ------------------------------------------------- a7, dense frames (BF16 GEMM)
 * Frames stored densely (uint16 counts, frames x P; no reference counterpart:
 * the reference stores photons sparsely, dset.py:23-60) go through the photon
 * term of calc_prob_all (kernels.cu:116-137) as a tensor-core GEMM:
 *   LL[r][d] = init[r / num_rot] * scale[d] + sum_c K[d][sel_pix[c]] L[r][c].
 *
 * rspi_dense_frames: K over the likelihood pixels as BF16 digit matrices
 * (frames x k_pad, K-major, zero beyond n_sel; k_pad % 64 == 0):
 * a0 = K & 255 and, when a1 != NULL, a1 = K - (K & 255); both exact in BF16.
 * *kmax (zeroed by the caller) gets the largest count; above 255 the caller
 * must pass a1. */
int rspi_dense_frames(const unsigned short *frames, long long n_frames, long long npix,
                      const int *sel_pix, long long n_sel, long long k_pad, void *a0, void *a1,
                      int *kmax, cudaStream_t stream);

/* Rotated log-slices of rows [row_begin, row_end) (the values of
 * rspi_rot_log_slices, computed in FP64) split into BF16 parts
 * hi = bf16(L), lo = bf16(L - hi), rows x k_pad each (zero beyond n_sel);
 * |L - hi - lo| <= 2^-16 |L|.  abs_max as in rspi_rot_log_slices. */
int rspi_rot_log_split(const double *holo, long long n_states0, long long num_rot,
                       const double *rot_cs, long long size, const double *bg,
                       const int *sel_pix, long long n_sel, long long k_pad,
                       long long row_begin, long long row_end, void *hi, void *lo,
                       float *abs_max, cudaStream_t stream);

/* Likelihood rows [row_begin, row_end) of every frame by tcgen05 BF16 MMAs
 * with FP32 accumulation in tensor memory: b_hi/b_lo hold n_brows slice rows
 * starting at row_begin; a1 may be NULL (counts below 256).  prob points at
 * row row_begin (row stride ld >= n_frames, frames contiguous, FP32).  All
 * matrix bases 16-byte aligned.  One call covers at most 65535 * 128 rows
 * (more is RSPI_ERR_ARG; split the range).  A device wait that exceeds its
 * bound sets *err = RSPI_ERR_TIMEOUT and leaves the tile's likelihoods
 * unwritten. */
int rspi_dense_loglike(const void *a0, const void *a1, const void *b_hi, const void *b_lo,
                       long long k_pad, long long n_frames, long long n_brows,
                       long long num_rot, long long row_begin, long long row_end,
                       const double *init, const double *scales, float *prob, long long ld,
                       int *err, cudaStream_t stream);

/* Exact integer variant of the dense likelihood (tcgen05 kind::i8): counts
 * as u8 (rspi_dense_frames_u8: frames x k_pad, k_pad % 128 == 0, counts
 * above 255 are clamped and *kmax tells the caller to use the BF16 path),
 * log-slices in fixed point Lq = rint(L * 2^21) as four 8-bit digit planes
 * (rspi_rot_log_fixed: rows [row_begin, row_end) into 4 planes of
 * plane_rows x k_pad bytes each, low digit first, the top one signed,
 * digits 4-byte aligned;
 * |L| >= 1023 or NaN is clamped and sets
 * *err = RSPI_ERR_CAPACITY), and rspi_dense_loglike_i8 accumulating each
 * digit product exactly in int32 (requires fewer than 8.4e6 photons per
 * frame on the likelihood pixels).  The only error of the photon term is
 * the quantisation, |err| <= 2^-22 * sum_p K[d][p]; the result goes to prob
 * as in rspi_dense_loglike (digits holds n_brows rows per plane). */
int rspi_dense_frames_u8(const unsigned short *frames, long long n_frames, long long npix,
                         const int *sel_pix, long long n_sel, long long k_pad, void *a,
                         int *kmax, cudaStream_t stream);

int rspi_rot_log_fixed(const double *holo, long long n_states0, long long num_rot,
                       const double *rot_cs, long long size, const double *bg,
                       const int *sel_pix, long long n_sel, long long k_pad,
                       long long row_begin, long long row_end, long long plane_rows,
                       void *digits, int *err, cudaStream_t stream);

int rspi_dense_loglike_i8(const void *a, const void *digits, long long k_pad,
                          long long n_frames, long long n_brows, long long num_rot,
                          long long row_begin, long long row_end, const double *init,
                          const double *scales, float *prob, long long ld, int *err,
                          cudaStream_t stream);

/* ----------------------------------------------------------------------- a16
 * Negative log-likelihood of the MaxLP model and its adjoint (no reference
 * counterpart works: get_grad_pixel, maxLP.py:199-214, uses an undefined
 * name).  Over the phaser pixels t (mask_idx[t] = m >= 0, qx/qy/qrad[m],
 * model fre/fim[m]) and frames d (rotation rot_cs[2d], rot_cs[2d+1] =
 * cos(-ang), sin(-ang); dia, sx, sy, scale):
 *   NLL = sum_d sum_t s_d |F_t + r_dt|^2 - k_dt log(s_d |F_t + r_dt|^2),
 *   r_dt = ff(pi qrad_t dia_d) exp(2 pi i (qx_t sx_d + qy_t sy_d)),
 * k_dt = photons of frame d at t's rotated pixel (maxLP.py:245-253).
 * precision 0: FP32 terms, 1: FP64 terms (sums always FP64).  With
 * want_grad the gradients d/dRe F, d/dIm F (n_pix) and d/d dia, sx, sy, scale
 * (n_frames) are written (zeroed first).  *nll is zeroed first. */
int rspi_nll(int precision, int want_grad, const int *ones, const int *multi,
             const long long *ones_accum, const long long *multi_accum, const int *place_ones,
             const int *place_multi, const int *count_multi, long long n_frames,
             const double *rot_cs, long long size, const int *mask_idx, long long n_pix,
             const double *fre, const double *fim, const double *qx, const double *qy,
             const double *qrad, const double *dia, const double *sx, const double *sy,
             const double *scale, double *nll, double *gfre, double *gfim, double *gdia,
             double *gsx, double *gsy, double *gscale, int *err, cudaStream_t stream);

/* The E-step side of the adjoint: negative log-likelihood through model
 * slicing for frames in given orientations (rot_cs[2d], rot_cs[2d + 1]: the
 * cos, sin of frame d's angle, as rspi_rot_log_slices uses them) with
 * continuous dia, sx, sy and scale per frame:
 *   NLL = sum_d [ vscale s_d sum_{q in sel} W_d(q)
 *                 - sum_{p in sel} K_d(p) (log s_d + L_d(p)) ]
 * W_d = |M + r_d|^2 + bg (slice_gen_holo, kernels.cu:58-75), L_d(p) the
 * bilinear rotated log-slice (slice_gen, kernels.cu:19-41; -1000, with no
 * gradient, outside the detector or below 1e-20): minus calc_prob_all's
 * value (kernels.cu:116-137, emc.py:194-199) with K_d log s_d added.
 * model complex128 size^2; sel_pix the n_sel likelihood pixels, pix2sel
 * their inverse map (-1 elsewhere).  With want_grad: gre/gim (size^2) and
 * gdia/gsx/gsy/gscale (n_frames) receive dNLL/d(Re M, Im M, dia, sx, sy, s).
 * precision 0: FP32 terms, 1: FP64; sums FP64.  No counterpart in the
 * reference, which has no gradient of its likelihood. */
int rspi_emc_nll(int precision, int want_grad, const double *model, long long size,
                 const double *bg, const int *sel_pix, long long n_sel, const int *pix2sel,
                 const int *ones, const int *multi, const long long *ones_accum,
                 const long long *multi_accum, const int *place_ones, const int *place_multi,
                 const int *count_multi, long long n_frames, const double *rot_cs,
                 const double *dia, const double *sx, const double *sy, const double *scale,
                 double vscale, double *nll, double *gre, double *gim, double *gdia,
                 double *gsx, double *gsy, double *gscale, int *err, cudaStream_t stream);

/* ------------------------------------------------------------ model refinement
 * Error reduction and difference map after the pattern search
 * (MaxLPhaser.proj_fourier / proj_real / er / diffmap / _get_support /
 * _improve_model, maxLP.py:271-298, 342-354).  Images are size x size
 * complex128 (row-major pixel t = x*size + y, 2 <= size <= 1024), masks one
 * byte per pixel (non-zero = true).  The centred transforms are NumPy's
 * fftshift(fftn(ifftshift(.))) and fftshift(ifftn(ifftshift(.))) as
 * line DFTs with the phase index reduced mod size in integer arithmetic.
 * work holds 8 * size^2 doubles.
 * rspi_cdft2: out = the centred forward (inverse = 0) or inverse (1) 2-D
 *   transform of in.
 * rspi_phase_support: minvsupp = !(G * |re(centred inverse of fconv *
 *   expit((mrad - taper_radius) * taper_slope))| > threshold), G the
 *   normalised Gaussian of `sigma` and half-width `radius` ('reflect'
 *   edges) along axis 0 then axis 1 (the reference: 12, 0.5, 3, 12, 1.2e-4).
 * rspi_phase_proj_fourier: out = x with the pixels of minvmask from fconv.
 * rspi_phase_proj_real: out = centred forward transform of the real part of
 *   the centred inverse transform of x, negatives and minvsupp pixels 0.
 * rspi_phase_refine: x <- n_dm difference-map steps
 *   x + proj_real(2 p - x) - p, p = proj_fourier(fconv, x), then n_er
 *   error-reduction steps x <- proj_real(proj_fourier(fconv, x)). */
int rspi_cdft2(const double *in, double *out, double *work, long long size, int inverse,
               cudaStream_t stream);
int rspi_phase_support(const double *fconv, long long size, double taper_radius,
                       double taper_slope, double sigma, int radius, double threshold,
                       unsigned char *minvsupp, double *work, cudaStream_t stream);
int rspi_phase_proj_fourier(const double *fconv, const unsigned char *minvmask, const double *x,
                            double *out, long long size, cudaStream_t stream);
int rspi_phase_proj_real(const double *x, const unsigned char *minvsupp, double *out,
                         double *work, long long size, cudaStream_t stream);
int rspi_phase_refine(const double *fconv, const unsigned char *minvmask,
                      const unsigned char *minvsupp, double *x, double *work, long long size,
                      int n_dm, int n_er, cudaStream_t stream);

/* ------------------------------------------------------------ data simulator
 * The per-frame loop of the reference's simulator (make_data.py:199-333),
 * batched: frames frame0 .. frame0 + n_frames - 1 of a dataset.
 * rspi_sim_views: view[f] (size^2 doubles per frame) = the holographic
 *   intensity scale[f] * |M_f + rel_scale * ff * ramp|^2 (kernels.cu:44-82,
 *   no background; ramp from shifts[2f], shifts[2f+1], ff from dia[f]) of the
 *   frame's model M_f, times mask_value on the detector mask (0 where
 *   r < 4 or r >= size/2; make_data.py:210-216 -- mask_value 2 for a
 *   heterogeneous object, whose two masks are added), scaled to sum to
 *   mean_count (make_data.py:316-318).  M_f by kind (make_data.py:294-309):
 *   0 iso: model; 1 homo, 2 mix, 3 blur: model plus wobble_model times the
 *   phase ramps e^{2 pi i w (qx + qy)} / e^{2 pi i w (qx - 3.7 qy)}
 *   (w = wobble[f]; mix alternates by the parity of frame0 + f; mirrored
 *   columns as np.fliplr).  model and wobble_model are complex128 size^2.
 *   A frame whose masked intensity sums to zero sets RSPI_ERR_ARG.
 * rspi_sim_counts: counts[f] (int32 size^2) ~ Poisson of the view rotated by
 *   the frame's angle (rot_cs[2f], rot_cs[2f+1] = cos, sin; slice_gen's
 *   bilinear rule, kernels.cu:6-42, pixels whose footprint leaves the
 *   detector 0) plus bg (NULL: none) on the others; expected (NULL: not
 *   written) receives the Poisson means.  Draws come from Philox4x32-10 with
 *   key = seed and counter (pixel, frame), so they do not depend on how the
 *   frames are batched.  n_frames <= 65535.  A mean that is negative, not
 *   finite or above 1e9 sets RSPI_ERR_ARG.
 * rspi_sim_poisson: out[i] ~ Poisson(lam[i]) from the same generator
 *   (stream_id separates the draws of different calls).
 * rspi_sim_sparse_counts: ones[f] / multi[f] = pixels of frame f with one /
 *   with more than one photon.
 * rspi_sim_sparse_fill: those pixels in ascending order at ones_off[f] /
 *   multi_off[f] (exclusive prefix sums of ones / multi), with the counts of
 *   the latter in count_multi (make_data.py:324-328). */
int rspi_sim_views(const double *model, const double *wobble_model, int kind, long long frame0,
                   long long n_frames, const double *wobble, const double *shifts,
                   const double *dia, const double *scale, double rel_scale, double mean_count,
                   double mask_value, int size, double *view, int *err, cudaStream_t stream);
int rspi_sim_counts(const double *view, long long frame0, long long n_frames,
                    const double *rot_cs, const double *bg, int size, unsigned long long seed,
                    int *counts, double *expected, int *err, cudaStream_t stream);
int rspi_sim_poisson(const double *lam, long long n, unsigned long long seed,
                     unsigned long long stream_id, int *out, int *err, cudaStream_t stream);
int rspi_sim_sparse_counts(const int *counts, long long n_frames, long long num_pix, int *ones,
                           int *multi, cudaStream_t stream);
int rspi_sim_sparse_fill(const int *counts, long long n_frames, long long num_pix,
                         const long long *ones_off, const long long *multi_off, int *place_ones,
                         int *place_multi, int *count_multi, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* RSPI_H */
