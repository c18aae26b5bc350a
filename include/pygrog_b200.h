/*
 * pygrog_b200.h -- C ABI of the sm_100a GROG gridding hot path.
 *
 * Every entry point takes plain device pointers, element counts and a
 * cudaStream_t (passed as void*), launches asynchronously on that stream,
 * allocates nothing, and returns a status code (PGB_OK == 0).  On failure,
 * pgb_last_error() returns a human-readable message for the calling thread.
 *
 * Complex data are interleaved (re, im) pairs: complex64 = float2,
 * complex128 = double2.  `dtype` selects PGB_C64 (complex64 data with float32
 * weights) or PGB_C128 (complex128 data with float64 weights).
 *
 * Reference interfaces replaced (FiRMLAB-Pisa/pygrog):
 *   csrc/torch/module.cpp:54-87 binds seven functions with pybind11; each
 *   pgb_* entry point below that carries a "replaces" line is its drop-in.
 *   The remaining entry points are the fused operators of the GROG path
 *   (plan build, fused grid/degrid, SparseFFT/Toeplitz pointwise stages and
 *   the device-side CG scalars), each citing the reference Python it
 *   replaces.
 */
#ifndef PYGROG_B200_H
#define PYGROG_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PGB_API __attribute__((visibility("default")))
#else
#define PGB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define PGB_OK 0
#define PGB_ERR_INVALID 1     /* bad size / shape / pointer               */
#define PGB_ERR_DTYPE 2       /* unsupported dtype code                   */
#define PGB_ERR_CUDA 3        /* kernel launch or CUDA runtime failure    */
#define PGB_ERR_UNSUPPORTED 4 /* e.g. coil count above the kernel limit   */
#define PGB_ERR_RANGE 5       /* index or size beyond a documented limit  */

/* ---- dtype codes ----------------------------------------------------- */
#define PGB_C64 0  /* complex64 data, float32 weights  */
#define PGB_C128 1 /* complex128 data, float64 weights */

/* Message for the last failing call on this host thread ("" if none). */
PGB_API const char* pgb_last_error(void);
/* Library version string. */
PGB_API const char* pgb_version(void);

/* =====================================================================
 * L0: the seven native functions of the reference extension
 * ===================================================================== */

/* out[n,b,co] = sum_ci kernel[idx[n],co,ci] * data[n,b,ci]
 * data (N,B,C), idx (N,) int64, kernel (K,C,C), out (N,B,C).
 * idx outside [0,K) yields zeros.
 * replaces: grog_interpolate, csrc/torch/grog_interp.cpp:112-149 and
 *           csrc/torch/grog_interp_cuda.cu:64-106 */
PGB_API int pgb_grog_interpolate(const void* data, const int64_t* idx, const void* kernel,
                         void* out, int64_t N, int64_t B, int64_t C, int64_t K,
                         int dtype, void* stream);

/* grid[idx[i]] += w[i] * data[i] (in place); indices outside [0,G) skipped.
 * Sorted indices are fastest but not required.
 * replaces: scatter_add, csrc/torch/sparse_ops.cpp:233-267,
 *           csrc/torch/sparse_ops_cuda.cu:47-63,149-173 */
PGB_API int pgb_scatter_add(void* grid, int64_t G, const void* data, const int64_t* idx,
                    const void* w, int64_t N, int dtype, void* stream);

/* Same result as pgb_scatter_add; uses the caller's bin layout
 * (bin_starts (n_bins+1,) int64 offsets into sorted idx, bins of bin_size
 * cells) to accumulate each bin in shared memory.
 * replaces: scatter_add_binned, csrc/torch/sparse_ops.cpp:299-340,
 *           csrc/torch/sparse_ops_cuda.cu:79-120,175-201 */
PGB_API int pgb_scatter_add_binned(void* grid, int64_t G, const void* data,
                           const int64_t* idx, const void* w, int64_t N,
                           const int64_t* bin_starts, int64_t n_bins,
                           int64_t bin_size, int dtype, void* stream);

/* out[i] = w[i] * grid[idx[i]] (0 for idx outside [0,G)).
 * replaces: gather, csrc/torch/sparse_ops.cpp:269-297,
 *           csrc/torch/sparse_ops_cuda.cu:126-143,203-230 */
PGB_API int pgb_gather(const void* grid, int64_t G, const int64_t* idx, const void* w,
               void* out, int64_t N, int dtype, void* stream);

/* psf[idx[i]] += w_sq[i] (real psf, float32 or float64 by dtype).
 * replaces: psf_scatter_scalar, csrc/torch/toep_psf.cpp:242-274,
 *           csrc/torch/toep_psf_cuda.cu:41-76 */
PGB_API int pgb_psf_scatter_scalar(void* psf, int64_t G, const int64_t* idx,
                           const void* w_sq, int64_t N, int dtype, void* stream);

/* psf[idx[i],l,l'] += w_sq[i] * conj(b[i,l]) * b[i,l']; psf (G,M,M) complex,
 * basis_per_sample (N,M) complex.
 * replaces: psf_scatter_outer, csrc/torch/toep_psf.cpp:276-323,
 *           csrc/torch/toep_psf_cuda.cu:83-133 */
PGB_API int pgb_psf_scatter_outer(void* psf, int64_t G, int64_t M, const int64_t* idx,
                          const void* w_sq, const void* basis_per_sample,
                          int64_t N, int dtype, void* stream);

/* psf[idx[i],k,k'] += w_sq[i] * conj(B[k,t_i]) * B[k',t_i]; psf (G,K,K),
 * basis (K,T), time_index (N,) int64 (outside [0,T) skipped).
 * replaces: psf_scatter_outer_basis, csrc/torch/toep_psf.cpp:325-367,
 *           csrc/torch/toep_psf_cuda.cu:138-193 */
PGB_API int pgb_psf_scatter_outer_basis(void* psf, int64_t G, int64_t K,
                                const int64_t* idx, const void* w_sq,
                                const void* basis, int64_t T,
                                const int64_t* time_index, int64_t N, int dtype,
                                void* stream);

/* =====================================================================
 * GROG plan construction (float32, bit-exact integer keys)
 * ===================================================================== */

/* Per-replica geometry of _create_plan_single (calib/_grog.py:1125-1212)
 * for one trajectory.  coords_scaled (npts, ndim) float32 are the rescaled
 * coordinates; offsets (kw, ndim) int32.  Writes, for r = n*kw + j:
 *   target_idx[r] int64 flat cell (-1 when out of bounds or |d|>0.5),
 *   distances[r*ndim + d] float32, gauss[r] float32 (0 when invalid).
 * grid_shape (int64), origins and grid_steps (float32) are per-axis HOST
 * arrays (ndim <= 3) read by the launcher; all other pointers are device
 * pointers. */
PGB_API int pgb_plan_geometry(const float* coords_scaled, int64_t npts, int ndim,
                      const int32_t* offsets, int kw, const int64_t* grid_shape,
                      const float* origins, const float* grid_steps,
                      int64_t* target_idx, float* distances, float* gauss,
                      void* stream);

/* gauss_sum[target] += (double)gauss (valid replicas); EGROG normalisation,
 * calib/_grog.py:1203-1206. */
PGB_API int pgb_plan_gauss_sum(const int64_t* target_idx, const float* gauss, int64_t R,
                       double* gauss_sum, int64_t G, void* stream);

/* weights[r] = gauss[r] / (float)max(gauss_sum[t], 1e-12) for valid r, else 0;
 * calib/_grog.py:1208-1212. */
PGB_API int pgb_plan_weights(const int64_t* target_idx, const float* gauss,
                     const double* gauss_sum, int64_t R, float* weights,
                     void* stream);

/* Shift quantisation of calc_interp_table (calib/_grog.py:406-417):
 *   i_d = rint((radius + rint(d*pfac)/pfac) / stepsize)
 *   idx = clamp(sum_d (int32) rint(i_d * nsteps^d), 0, K-1)
 * all in float32 with IEEE division (pfac, stepsize given as float32). */
PGB_API int pgb_plan_quantize(const float* distances, int64_t R, int ndim, float radius,
                      float pfac, float stepsize, int nsteps, int64_t K,
                      int64_t* interp_idx, void* stream);

/* Host-side packing steps of the brick plans of the fused gridders (host
 * pointers, no device work; sequential per sub-chunk, threaded over
 * sub-chunks).  No reference counterpart: the reference computes every
 * replica unbinned (calib/_grog.py:1283-1295); these lay the binned replicas
 * out for the kernels below.
 *
 * pgb_plan_pack_quarter_warps: sub-chunk s holds replicas
 * [sub_ptr[s], sub_ptr[s + 1]) in processing order with inner / outer table
 * indices q / k; every replica gets lane = quarter_warp * per + slot, packing
 * nq[s] = ceil(count / per) quarter-warps first-fit: a replica goes to the
 * first quarter-warp with a free lane that already reads its inner operator,
 * else has its inner residue class (q mod per) free, both with a compatible
 * outer residue (k mod per: free or the same k), else has a compatible inner
 * residue, else has the fewest lanes taken.  per = 8 or 4.
 *
 * pgb_plan_pack_rows: sub-chunk s holds cell runs [run_ptr[s], run_ptr[s+1])
 * of run_len entries; runs are laid out in order from entry 0, a run of at
 * most `rows` entries that would cross a multiple of `rows` starts at the
 * next one (padding entries in between) as long as the sub-chunk's entries
 * stay within `cap`; run_start gets each run's first entry, n_entries[s] the
 * sub-chunk's entries including padding.
 *
 * pgb_plan_lpt: item i of cost[i] goes to out[i] in [0, bins): items in
 * decreasing cost (ties in index order), each to the least loaded bin (ties
 * to the lowest bin). */
PGB_API int pgb_plan_pack_quarter_warps(const int64_t* sub_ptr, const int64_t* q, const int64_t* k,
                                        int64_t n_subs, int64_t per, int64_t* lane, int64_t* nq);
PGB_API int pgb_plan_pack_rows(const int64_t* run_len, const int64_t* run_ptr, int64_t n_subs, int64_t rows,
                               int64_t cap, int64_t* run_start, int64_t* n_entries);
PGB_API int pgb_plan_lpt(const double* cost, int64_t n, int64_t bins, int32_t* out);

/* =====================================================================
 * Fused GROG operator (interpolate + weight + scatter, and its adjoint)
 * ===================================================================== */

/* Brick work plan shared by the fused kernels.  Valid replicas are sorted
 * by (brick, cell); per replica:
 *   rep_src  int32   source sample index,
 *   rep_meta uint32  table entry (low 20 bits) | cell-in-brick << 20,
 *   rep_w    float32 replica weight.
 * work (n_work, 4) int32 rows: {brick, begin, end, split}; split=1 marks a
 * chunk of a brick shared by several chunks.  Bricks are (bz,by,bx) cells
 * (2-D grids use bz=1, grid_shape[0]=1). */
typedef struct pgb_brick_plan {
  const int32_t* rep_src;
  const uint32_t* rep_meta;
  const float* rep_w;
  const int32_t* work;
  int32_t n_work;
  int32_t gz, gy, gx;       /* grid extent per axis (2-D: gz = 1)      */
  int32_t bz, by, bx;       /* brick extent per axis                   */
  int32_t nbz, nby, nbx;    /* bricks per axis                         */
  const int32_t* split_bricks; /* bricks touched by split chunks     */
  int32_t n_split_bricks;
} pgb_brick_plan;

/* Forward: grid[b,c,cell] = sum_{r->cell} w_r * (T[e_r] @ data[b,:,src_r])[c]
 * data (B,C,N) complex64, grid (B,C,G) complex64, table (K,C,C) complex64.
 * Every grid cell is written.  Replaces interpolate(grid=True),
 * calib/_grog.py:437-555,668-695,736-902 (replicate, grog_interpolate,
 * pre_weights, per-coil scatter_add). C <= 32. */
PGB_API int pgb_grog_grid(const void* data, int64_t N, void* grid, int64_t G,
                  const void* table, int64_t K, int64_t C, int64_t B,
                  const pgb_brick_plan* plan, void* stream);

/* Adjoint: out[b,:,n] = sum_{r: src_r=n} w_r * T[e_r]^H @ grid[b,:,cell_r]
 * table_h (K,C,C) holds the conjugate transposes of the table.
 * `accumulate` = 0 when every sample has at most one valid replica (plain
 * stores; samples listed in zero_src (n_zero) are zeroed), 1 otherwise
 * (out is zeroed then accumulated atomically).  No reference counterpart:
 * the G^H adjoint of interpolate(grid=True) restated from its definition. */
PGB_API int pgb_grog_degrid(const void* grid, int64_t G, void* out, int64_t N,
                    const void* table_h, int64_t K, int64_t C, int64_t B,
                    const pgb_brick_plan* plan, int accumulate,
                    const int32_t* zero_src, int64_t n_zero, void* stream);

/* Operator-stationary variants (C <= 16, power-of-two bricks of at most
 * 4096 cells).  Replaces the per-replica operator application of
 * calib/_grog.py:1283-1295 fused with the scatter of
 * operator/_sparse_fft.py:416 (forward) and its adjoint.
 *
 * Plan layout (device arrays, built by pygrog_b200.calib.BrickPlan6):
 *   sd[]        int4 {rep_begin, rep_end, uniq_begin, uniq_end} per sub-chunk,
 *               grouped per CTA in processing order (CTA c owns entries
 *               cta_ptr[c] .. cta_ptr[c+1]-1; launch uses n_cta CTAs)
 *   si[]        int2 {brick, flags}: 1 first sub-chunk of a brick item,
 *               2 last one (flush), 4 the brick is split over several items
 *   uniq[]      int32 source sample of every staging slot, ascending inside
 *               a sub-chunk (at most sub_cap <= 512 slots / replicas each)
 *   meta[]      int2 {cell | slot << 16, inner | outer << 16} per replica
 *   w[]         float weight per replica
 *   zero_bricks bricks the forward writes with zeros first (empty + split);
 *               the last n_empty_tail of them are empty bricks (no
 *               sub-chunk touches them), which the tensor-core forward on
 *               its tensor-copy path clears from inside its kernel while
 *               it grids (0: every listed brick is cleared beforehand)
 * inner_lc / outer_lc (forward) and inner_h_lc / outer_h_lc (adjoint): the
 * factors (inner = whole table when n_outer == 1; outer unused then) in
 * lane-chunk layout, entry (q, j, l, t) = M[q][l*RPL + t][j] with RPL = 2
 * for even C (else 1) and L = C / RPL; M = inner / outer for the forward,
 * their conjugate transposes for the adjoint.
 * Shared memory: pgb_grog_v6_smem_bytes(C, cells, n_inner, n_outer, sub_cap). */
typedef struct pgb_v6_plan {
  const int32_t* sd;
  const int32_t* si;
  const int32_t* cta_ptr;
  int32_t n_cta;
  const int32_t* uniq;
  const int32_t* meta;
  const float* w;
  int32_t sub_cap;
  int32_t gz, gy, gx;
  int32_t bz, by, bx;
  int32_t nbz, nby, nbx;
  const int32_t* zero_bricks;
  int32_t n_zero_bricks;
  /* cell order of every sub-chunk, for the lane-per-replica forward (may be
   * NULL otherwise): entry = pos | cell << 9 | head << 21 | shared << 22,
   * sorted by (cell, pos) inside the sub-chunk, pos = index of the replica in
   * it; a head starts a segment of entries of one cell (summed by one thread),
   * shared marks segments of a cell that has several (added atomically) */
  const int32_t* cword;
  int32_t n_empty_tail;
} pgb_v6_plan;

PGB_API size_t pgb_grog_v6_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int64_t n_outer,
                                      int64_t sub_cap);
PGB_API int pgb_grog_grid_v6(const void* data, int64_t N, void* grid, int64_t G, const void* inner_lc,
                             int64_t n_inner, const void* outer_lc, int64_t n_outer, int64_t C, int64_t B,
                             const pgb_v6_plan* plan, void* stream);
/* primary: every sample at most once (plain stores); secondary (may be NULL):
 * the remaining replicas (atomic adds); zero_src: samples with no replica. */
PGB_API int pgb_grog_degrid_v6(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h_lc,
                               int64_t n_inner, const void* outer_h_lc, int64_t n_outer, int64_t C, int64_t B,
                               const pgb_v6_plan* primary, const pgb_v6_plan* secondary,
                               const int32_t* zero_src, int64_t n_zero, void* stream);

/* One-lane-per-replica variants on the v6 plan (C <= 16; plan sub_cap <= 256:
 * one replica per thread of a 256-thread CTA; any replica order inside a
 * sub-chunk is correct, the quarter-warp packing of the plan only removes
 * bank conflicts; entries with meta.x < 0 are padding).  The forward needs
 * the plan's cell order (cword).  inner / outer (forward) and inner_h /
 * outer_h (adjoint): row-major (n, C, C) operators (inner = whole table when
 * n_outer == 1).  Same contract as pgb_grog_grid_v6 / pgb_grog_degrid_v6.
 * Shared memory: pgb_grog_v8_smem_bytes(C, cells, n_inner, n_outer, sub_cap). */
PGB_API size_t pgb_grog_v8_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int64_t n_outer,
                                      int64_t sub_cap);
PGB_API int pgb_grog_grid_v8(const void* data, int64_t N, void* grid, int64_t G, const void* inner,
                             int64_t n_inner, const void* outer, int64_t n_outer, int64_t C, int64_t B,
                             const pgb_v6_plan* plan, void* stream);
PGB_API int pgb_grog_degrid_v8(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h,
                               int64_t n_inner, const void* outer_h, int64_t n_outer, int64_t C, int64_t B,
                               const pgb_v6_plan* primary, const pgb_v6_plan* secondary,
                               const int32_t* zero_src, int64_t n_zero, void* stream);
/* Tensor-core (mma.sync bf16, fp32 accumulate) gridding: the same operator as
 * the table path of calib/_grog.py:1283-1295 + operator/_sparse_fft.py:416
 * (forward) and its adjoint, with the table applied in its exact eigen-factored
 * form T = V2 D2[k] V2^-1 V1 D1[j] V1^-1 V0 D0[i] V0^-1 (calib/_grappa.py:62-72,
 * 130-208: every per-axis operator is expm(d logm G)).  wfrag: int32
 * (ndim + 1, 2, NFR, 32) bf16x2 head / tail B-fragment words of the dense
 * stages in application order (calib/_tc.py), NFR = (CP/4) * (CP/4 rounded
 * down to even + (CP/4) % 2), CP = C rounded up to a multiple of 4; dtab:
 * complex64 (ndim, nsteps, CP) diagonal phases in application order.  terms: 3
 * = bf16x3 split products (~1e-5 relative), 1 = plain bf16.  Plans: v6 plans
 * built with n_outer = nsteps,
 * sub_cap <= 256, meta.y = the per-axis shift indices (3-D i | j << 8 | k << 16
 * with e = (i nsteps + j) nsteps + k and nsteps <= 255; 2-D i | k << 16 with
 * e = i nsteps + k); the forward plan in (cell, sample) order inside each
 * sub-chunk with meta.x bit 30 set on cells whose run crosses a 16-entry
 * boundary; C <= 16.  The plan's n_cta should be 148 x
 * pgb_grog_tc_blocks_per_sm(C, ndim).  Same zeroing / primary / secondary /
 * zero_src contract as pgb_grog_grid_v6 / pgb_grog_degrid_v6. */
PGB_API size_t pgb_grog_tc_smem_bytes(int64_t C, int64_t cells, int64_t nsteps, int64_t ndim, int64_t sub_cap);
PGB_API int pgb_grog_tc_blocks_per_sm(int64_t C, int64_t ndim);
PGB_API int pgb_grog_grid_tc(const void* data, int64_t N, void* grid, int64_t G, const void* wfrag,
                             const void* dtab, int64_t nsteps, int64_t ndim, int64_t C, int64_t B, int64_t terms,
                             const pgb_v6_plan* plan, void* stream);
PGB_API int pgb_grog_degrid_tc(const void* grid, int64_t G, void* out, int64_t N, const void* wfrag_h,
                               const void* dtab_h, int64_t nsteps, int64_t ndim, int64_t C, int64_t B,
                               int64_t terms, const pgb_v6_plan* primary, const pgb_v6_plan* secondary,
                               const int32_t* zero_src, int64_t n_zero, void* stream);
/* Brick tiles of the tensor-core gridder move by tensor-memory-accelerator
 * copies (one bulk tensor load / store / reduce-add per brick, mbarrier
 * completion) when the grid allows it (even gx and brick width, 16-byte
 * aligned grid, C a multiple of 4); otherwise by per-element async copies.
 * pgb_grog_tc_use_tma(0 / 1) turns the tensor copies off / on for later calls
 * (negative: query only) and returns the previous setting.  No reference
 * counterpart (performance switch). */
PGB_API int pgb_grog_tc_use_tma(int64_t enable);
/* Number of tile waits that gave up (bounded mbarrier spin; the CTA then
 * lets its copies in flight land and returns without writing the rest of its
 * results); reset when reset != 0.  Synchronous.  The Python layer raises
 * RuntimeError when it reads a non-zero count.  No reference counterpart
 * (diagnostics). */
PGB_API int pgb_grog_tc_timeouts(int64_t* count, int64_t reset);
/* Spin limit of the adjoint's tile waits for later launches (limit >= 0;
 * -1 restores the default of 2^26 polls); the previous limit goes to
 * *previous when it is non-null.  Synchronous.  A limit of 0 makes every
 * tile wait give up at once, which exercises the timeout path without any
 * fault: the copies still complete and are drained before the CTA exits.
 * No reference counterpart (failure-path testing). */
PGB_API int pgb_grog_tc_wait_limit(int64_t limit, int64_t* previous);

/* The eigen-factored shift chain alone, y = W3 Dx[k] W2 Dy[j] W1 Dz[i] W0 x on
 * R replicas (the table product of calib/_grappa.py:62-72, 184-208 applied to
 * one replica, as the tensor-core gridders run it), in two tensor-core forms,
 * for measuring the MMA flavour: variant 0 = mma.sync with the accumulators
 * handed on in registers, variant 1 = tcgen05.mma with the accumulator in
 * tensor memory (M = 128 replicas per tile).  bf16x3 products, FP32
 * accumulation.  C = 12 or 32 coils.  x, out: (2C, R) float realified
 * (row 2c real part of coil c, 2c + 1 imaginary); idx: R int32
 * i | j << 8 | k << 16, each < 11 (a larger byte reads step 10); W: (4, 2C, 2C) float realified
 * [stage][output][input]; ph: (3, 11, C) complex64 phases.  rep >= 1 applies
 * the chain rep times per loaded tile.  timeouts: int32 device counter
 * (required for variant 1), incremented by every CTA whose bounded tensor-core
 * waits ran out.  Asynchronous on `stream`.  No reference counterpart. */
PGB_API int pgb_shift_chain(const void* x, const void* idx, const void* W, const void* ph, void* out, int64_t R,
                            int64_t C, int64_t rep, int64_t variant, void* timeouts, void* stream);

/* =====================================================================
 * Coil compression (the step before the path)
 * ===================================================================== */

/* cov (C, C) complex128 <- sum_m data[i, m] conj(data[j, m]) over the M
 * samples of data (C, M) complex64 (coil-major), accumulated in FP64.  The
 * covariance whose leading eigenvectors are the compression matrix of
 * replaces: utils/_coil_compress.py:23-57 (coil_compress, which forwards to
 * mrinufft's coil_compression).  C <= 32. */
PGB_API int pgb_coil_covariance(const void* data, int64_t M, int64_t C, void* cov, void* stream);
/* cov (C, C) complex128 <- sum_m data[i, m] conj(data2[j, m]) (FP64): the
 * Gram matrices of the Tikhonov least squares of the unit GROG operators,
 * src^H src and src^H dst over neighbour pairs of the calibration block
 * (replaces the O(samples) part of calib/_grappa.py:16-59, lstsq, in the GPU
 * table fit).  C <= 32. */
PGB_API int pgb_coil_cross_covariance(const void* data, const void* data2, int64_t M, int64_t C, void* cov,
                                      void* stream);
/* out (B, K, N) complex64 <- mat (K, C) complex64 @ data (B, C, N): the
 * compression step of the same function.  1 <= K <= C <= 64. */
PGB_API int pgb_coil_compress(const void* data, int64_t N, int64_t C, int64_t K, int64_t B, const void* mat,
                              void* out, void* stream);
/* The same product on the tensor cores (mma.sync bf16x3, FP32 accumulate,
 * ~1e-5 relative): the matrix as register-resident A fragments, 8 samples x
 * all coils per B fragment.  1 <= K <= min(C, 16), C <= 32. */
PGB_API int pgb_coil_compress_tc(const void* data, int64_t N, int64_t C, int64_t K, int64_t B, const void* mat,
                                 void* out, void* stream);

/* Replica expansion of interpolate() (calib/_grog.py:668-695):
 * out[b,co,n*kw+j] = sum_ci T[interp_idx[n*kw+j],co,ci] * data[b,ci,n]
 * data (B,C,N), out (B,C,N*kw); entries outside [0,K) give 0. C <= 32. */
PGB_API int pgb_grog_expand(const void* data, int64_t N, int kw, const int64_t* interp_idx,
                    const void* table, int64_t K, int64_t C, int64_t B, void* out,
                    void* stream);

/* =====================================================================
 * SparseFFT / MaskedFFT / Toeplitz stages around cuFFT
 * (operator/_sparse_fft.py:574-621, 741-789, 1154-1177;
 *  operator/_masked_fft.py:322-430; _toep/_grog_toep.py:154-209;
 *  _base/_fftc.py:114-139)
 * Buffers handed to cuFFT are in "FFT order": centred grid index p (per
 * axis, extent g) is stored at m = (p - g/2) mod g, which is exactly
 * ifftshift, so no shift pass is ever made.  grid_shape / image_shape are
 * HOST arrays of ndim (2 or 3) extents; all other pointers are device
 * pointers; complex data are complex64.
 * ===================================================================== */

/* u[b,c,m] = scale * S[c,q(m)] * x[b,q(m)] (x_has_coils = 0, smaps may be
 * NULL for a single coil) or scale * x[b,c,q(m)] (x_has_coils = 1); zero
 * outside the centred image: zero-pad + coil expansion + ifftshift. */
PGB_API int pgb_fft_expand(const void* x, const void* smaps, void* u, int64_t B, int64_t C,
                           int ndim, const int64_t* grid_shape, const int64_t* image_shape,
                           float scale, int x_has_coils, void* stream);

/* out[b,q] = scale * sum_c conj(S[c,q]) v[b,c,m(q)] (smaps) or
 * out[b,c,q] = scale * v[b,c,m(q)] (smaps NULL); plus add_scale * add[...]
 * when add is not NULL: fftshift + crop + coil combine (+ damping term). */
PGB_API int pgb_fft_combine(const void* v, const void* smaps, void* out, int64_t B, int64_t C,
                            int ndim, const int64_t* grid_shape, const int64_t* image_shape,
                            float scale, const void* add, float add_scale, void* stream);

/* u[bc, cellpos[r]] += w[r] * data[bc, r] for bc < BC (u pre-zeroed by the
 * caller); entries with cellpos outside [0,G) or w == 0 are skipped. */
PGB_API int pgb_sparse_scatter(const void* data, const int32_t* cellpos, const float* w, void* u,
                               int64_t BC, int64_t R, int64_t G, void* stream);

/* out[bc, r] = w[r] * U[bc, cellpos[r]] (0 for cellpos outside [0,G)). */
PGB_API int pgb_sparse_gather(const void* U, const int32_t* cellpos, const float* w, void* out,
                              int64_t BC, int64_t R, int64_t G, void* stream);

/* Low-rank subspace transfers (replace the per-(coil, component) scatter /
 * gather loops of gadgets/_subspace.py:311-508 and the PSF matvec of
 * _toep/_sub_toep.py:236-303).  y (B, C, R) natural sample order, u / U
 * (B, K, C, G) FFT-order grids, basis (K, T) complex64, tidx (R) int32 index
 * along the encoding axis, cellpos (R) int32 FFT-order cell, w (R) float.
 *   scatter: u[b,k,c,cell_r] += w_r * basis[k,t_r] * y[b,c,r]
 *   gather:  y[b,c,r] = w_r * sum_k conj(basis[k,t_r]) * U[b,k,c,cell_r]
 *   psf_apply_kk (in place): U[b,k,c,g] = sum_k' P[g,k,k'] * U[b,k',c,g],
 *            P (G, K, K) complex64, K <= 16. */
PGB_API int pgb_subspace_scatter(const void* y, const int32_t* cellpos, const float* w, const int32_t* tidx,
                                 const void* basis, void* u, int64_t B, int64_t C, int64_t K, int64_t T,
                                 int64_t R, int64_t G, void* stream);
PGB_API int pgb_subspace_gather(const void* U, const int32_t* cellpos, const float* w, const int32_t* tidx,
                                const void* basis, void* out, int64_t B, int64_t C, int64_t K, int64_t T,
                                int64_t R, int64_t G, void* stream);
PGB_API int pgb_psf_apply_kk(void* U, const void* P, int64_t B, int64_t K, int64_t C, int64_t G, void* stream);

/* U[bc, m] *= psf[m] (real PSF in FFT order; Toeplitz normal operator). */
PGB_API int pgb_psf_apply(void* U, const float* psf, int64_t BC, int64_t G, void* stream);

/* to_centred = 0: dst[bc,m] = scale * mask[p(m)] * src[bc,p(m)];
 * to_centred = 1: dst[bc,p] = scale * mask[p] * src[bc,m(p)]  (mask may be
 * NULL).  src and dst must not alias. */
PGB_API int pgb_fft_shift(const void* src, const float* mask, void* dst, int64_t BC, int ndim,
                          const int64_t* grid_shape, float scale, int to_centred, void* stream);

/* =====================================================================
 * Conjugate gradient scalars in FP64 on the device (_solve/_solvers.py:49-139)
 * scalars: double[8] = {rz_old, pAp, rr, r0_norm, rel, done, tol, spare}
 * scratch: pgb_reduce_scratch_bytes() bytes, zero-initialised once; its
 * counters return to zero after every call.  Every kernel is a no-op once
 * done != 0, which replaces the host-side early exit.
 * ===================================================================== */
PGB_API size_t pgb_reduce_scratch_bytes(void);
/* mode 0: scalars[out_slot] = sum Re(conj(a) b) (b NULL: |a|^2);
 * mode 1: rr = |a|^2, rel = sqrt(rr)/r0_norm, done |= rel < tol;
 * mode 2: CG start: rr = rz_old = |a|^2, r0_norm = sqrt(rr) + 1e-30. */
PGB_API int pgb_dot_f64(const void* a, const void* b, int64_t n, void* scratch, void* scalars,
                        int out_slot, int mode, void* stream);
/* alpha = rz_old / (pAp + 1e-30); x += alpha p; r -= alpha Ap */
PGB_API int pgb_cg_update_xr(void* x, void* r, const void* p, const void* Ap, int64_t n,
                             const void* scalars, void* stream);
/* pgb_cg_update_xr followed by pgb_dot_f64(r, NULL, mode 1) in one pass:
 * x += alpha p; r -= alpha Ap; rr = |r|^2 (FP64), rel, done.  Uses the
 * scratch's first counter, as pgb_dot_f64 does. */
PGB_API int pgb_cg_update_xr_rr(void* x, void* r, const void* p, const void* Ap, int64_t n, void* scalars,
                                void* scratch, void* stream);
/* beta = rr / (rz_old + 1e-30); p = r + beta p; rz_old = rr */
PGB_API int pgb_cg_update_p(void* p, const void* r, int64_t n, void* scalars, void* scratch,
                            void* stream);
/* Frame-batched forms of the three CG kernels for `frames` independent
 * systems solved together (_solve/_solvers.py:49-139 run once per frame):
 * vectors are (frames, n) contiguous, scalars (frames, 8) doubles with the
 * layout above, scratch frames * pgb_reduce_scratch_bytes() bytes
 * (zero-initialised once).  Each frame keeps its own alpha, beta, residual
 * and done flag. */
PGB_API int pgb_dot_f64_batched(const void* a, const void* b, int64_t n, int64_t frames, void* scratch,
                                void* scalars, int out_slot, int mode, void* stream);
PGB_API int pgb_cg_update_xr_batched(void* x, void* r, const void* p, const void* Ap, int64_t n,
                                     int64_t frames, const void* scalars, void* stream);
PGB_API int pgb_cg_update_xr_rr_batched(void* x, void* r, const void* p, const void* Ap, int64_t n,
                                        int64_t frames, void* scalars, void* scratch, void* stream);
PGB_API int pgb_cg_update_p_batched(void* p, const void* r, int64_t n, int64_t frames, void* scalars,
                                    void* scratch, void* stream);
/* y += a x */
PGB_API int pgb_axpy(void* y, const void* x, float a, int64_t n, void* stream);

/* =====================================================================
 * LSMR with device-resident FP64 scalars.
 * replaces: _solve/_solvers.py:145-262 (lsmr: Golub-Kahan step, rotations
 * Q_k / Qbar_k, h / hbar / x updates, stopping test |zetabar| / |b| <
 * atol + btol), whose norms are FP32 and whose branches and stopping test
 * are host .item() reads.
 *
 * Scalar block: double[PGB_LSMR_SCALARS] in device memory, slots
 *   0 alpha  1 beta  2 alphabar  3 rho  4 rhobar  5 cbar  6 sbar  7 zetabar
 *   8 zeta  9 normb  10 stop  11 tol (atol + btol)  12 damp  13-15 the
 *   hbar / x / h update coefficients  16 |u|^2  17 |v_full|^2  18 ran
 *   19 rel  20 v updated  21 iterations.
 * The caller initialises slots 0-12 (Fong & Saunders' start: alpha, beta =
 * |b|, alphabar = alpha, rho = rhobar = cbar = 1, sbar = 0, zetabar =
 * alpha beta, normb = beta, stop = 0) and runs per iteration, on one stream:
 *   Av = A v;  pgb_lsmr_u_update(u, Av);  pgb_lsmr_u_scale(u);
 *   Atu = A^H u;  pgb_lsmr_v_full(vf, Atu, v);  pgb_lsmr_scalars;
 *   pgb_lsmr_vec_update(x, h, hbar, v, vf).
 * Norms accumulate in FP64; vectors are complex64.  Once the stopping test
 * has fired every later call leaves vectors and scalars unchanged, so a
 * captured iteration can be replayed max_iter times.  scratch holds
 * pgb_lsmr_scratch_bytes() bytes, zero-initialised once; calls that share a
 * scratch must be ordered on one stream. */
#define PGB_LSMR_SCALARS 32
PGB_API size_t pgb_lsmr_scratch_bytes(void);
/* u <- Av - alpha u ; slot 16 <- |u|^2 */
PGB_API int pgb_lsmr_u_update(void* u, const void* Av, int64_t n, void* scal, void* scratch, void* stream);
/* u <- u / sqrt(slot 16) when slot 16 > 0 */
PGB_API int pgb_lsmr_u_scale(void* u, int64_t n, const void* scal, void* stream);
/* vf <- Atu - beta v (beta = sqrt(slot 16)) ; slot 17 <- |vf|^2 ; only when slot 16 > 0 */
PGB_API int pgb_lsmr_v_full(void* vf, const void* Atu, const void* v, int64_t n, void* scal, void* scratch,
                            void* stream);
/* the scalar recurrence of one iteration (one thread) */
PGB_API int pgb_lsmr_scalars(void* scal, void* stream);
/* v <- vf / alpha (when updated) ; hbar <- h - c1 hbar ; x <- x + c2 hbar ; h <- v - c3 h */
PGB_API int pgb_lsmr_vec_update(void* x, void* h, void* hbar, void* v, const void* vf, int64_t n,
                                const void* scal, void* stream);

/* =====================================================================
 * Allocation-free row inner products.  No counterpart in the reference
 * (FiRMLAB-Pisa/pygrog has no C entry point of this kind; its solvers call
 * torch.vdot, _solve/_solvers.py:49-139).
 *
 * out[r] = sum_i Re(conj(a[r, i]) b[r, i])   (b NULL: sum_i |a[r, i]|^2),
 * accumulated in FP64, for `rows` contiguous complex64 vectors of n
 * elements; out is a device array of `rows` doubles.  Same arithmetic as
 * pgb_dot_f64 mode 0, one vector per row.
 *
 * For callers that must not allocate device memory while they run: code
 * working inside a fixed, pre-reserved memory budget (a reconstruction
 * service whose pool is fully handed out), real-time loops where an
 * allocation may block or fail, and bindings from languages with no access
 * to a device allocator.  Its scratch (block partials and completion
 * counters, 151,808 bytes) is a static array inside this library, so
 * nothing is allocated or freed by the call.
 *
 * Limit: rows <= 64; larger rows return PGB_ERR_RANGE with a message.
 * The first call on each device looks up the scratch address (with that
 * device current) and caches it together with the current context; a call
 * that finds another context current (after cudaDeviceReset, say) looks the
 * address up again.  Make the first call on a device, and the first one
 * after a reset, before any stream capture.  Every call clears the counters it uses on `stream` before its
 * kernel runs.  All calls on one device share the one scratch array, so
 * calls that can overlap on the GPU (different streams without ordering
 * between them) race and give wrong results: order them on one stream. */
PGB_API int pgb_dot_f64_noalloc(const void* a, const void* b, int64_t n, int64_t rows, double* out,
                                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYGROG_B200_H */
