/*
 * lds.h — C ABI of liblds.so, the B200 implementation of SUMMIT's genotype x
 * probe hot path (BED decode, X.W and X^T.(X.W) over probe blocks with
 * on-the-fly centering and scaling, and the LD-score reductions on top).
 *
 * The reference exposes this path as nanobind Python functions (module
 * `gwldcore`, src/native/gwldcore.cpp:3656-3829).  Each entry point below is
 * the plain-C counterpart of one of them: host pointers and sizes, no Python
 * or torch types.  Arrays keep the reference's layouts:
 *   - Xz2d / Geno / C / R: column-major (Fortran order);
 *   - annot_blk, meansq_accum, mc_per_snp_sumsq: row-major (C order);
 *   - `_f32` / `_f64` suffixes select float32 / float64 arrays, like the
 *     nanobind overloads.
 * Optional arrays are passed as NULL.  Optional integers (seed, impute_seed)
 * come with a `has_` flag.  Every function returns 0 on success and a
 * negative code on failure; lds_last_error() then holds the message, which
 * the Python shim raises as RuntimeError (the reference raises
 * std::runtime_error -> RuntimeError with the same wording where it has one).
 *
 * Computation runs on the current CUDA device.  There is no CPU fallback:
 * without a usable device every compute entry returns LDS_ERR_CUDA.
 */
#ifndef LDS_H
#define LDS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDS_OK 0
#define LDS_ERR_ARG -1
#define LDS_ERR_CUDA -2
#define LDS_ERR_IO -3
#define LDS_ERR_INTERNAL -4

/* Probe distributions (gwldcore.cpp:1693-1716). */
#define LDS_DIST_RADEMACHER 0
#define LDS_DIST_GAUSSIAN 1
#define LDS_DIST_SPHERICAL 2

/* Imputation modes (genotype.hpp:33-36, ImputeMode). */
#define LDS_IMPUTE_MEAN 0
#define LDS_IMPUTE_HWE 1

/* Thread-local text of the last error. */
const char* lds_last_error(void);

/* Library build information ("liblds <version> sm_100a ..."). */
const char* lds_version(void);

/* Number of visible CUDA devices (0 when no driver/device). */
int lds_device_count(void);

/* Number of int8 digit slices used for floating operands (3..6, default 4).
 * Higher = closer to FP64 at proportional tensor-core cost. */
int lds_set_slices(int slices);
int lds_get_slices(void);

/* Guard counts of the last per-block phase-2 call on this process's
 * context: out2[0] = non-finite updates dropped, out2[1] = finite updates
 * above the extreme-LD threshold (dropped unless SUMMIT_P2_DROP_EXTREME=0).
 * The reference prints the same two counts per call
 * (phase2_log_guard_counts, gwldcore.cpp:364-417). */
int lds_phase2_guard_counts(uint64_t* out2);

/* Bounded waits.  Every wait of the tensor-core kernels on an mbarrier gives
 * up after `iters` tries (each suspends the thread for at most 200 ns;
 * default 2^25, about 6.7 s), records an error status and lets the kernel
 * return, so a stalled pipeline surfaces as LDS_ERR_CUDA instead of a hung
 * GPU.  lds_set_wait_limit applies to the current device and waits for the
 * library's work in flight; lds_get_wait_limit returns the value last set.
 * No counterpart in the reference (its CPU loops have no device waits). */
int lds_set_wait_limit(long long iters);
long long lds_get_wait_limit(void);
/* Self-test of the bounded wait: one thread waits on an mbarrier that nothing
 * arrives at, under the current limit.  *status_out = 1 when the wait ran
 * out and the kernel returned its error status (the expected result), 2 if
 * the wait completed. */
int lds_selftest_wait_timeout(unsigned* status_out);

/* Counters of the library's own CUDA kernel launches since process start
 * (all kernels) — used to report launches inside timed regions. */
uint64_t lds_kernel_launches(void);

/* Release cached device genotype images and workspaces
 * (clear_gwld_native_scratch, gwldcore.cpp:194-200; _clear_bed_mapping_cache,
 * :3668). */
void lds_clear_device_cache(void);

/* ---------------------------------------------------------------------
 * Phase 1: Xz2d[:, k*v_count+c] (+)= sum_{j in bin k} x_j * z_jc * inv_j*sqrt(a_jk)
 * for SNP block [blk_start, blk_end) of a PLINK BED fileset.
 * Replaces gwldcore.phase1_compute_Xz_bed_chunk (gwldcore.cpp:3673-3688,
 * implementation :1582-1894).  Xz2d is N x (K*v_count), column-major,
 * updated in place; bin_init_mask (K bytes, may be NULL) selects beta = 0
 * for a bin's first write and is set to 1 for bins written.  When inv_out is
 * given, residual variances of the block are computed into it and used in
 * place of inv_right (fused residual variance, :1659-1669).
 * Covariates enter only the fused residual variances, as in the reference's
 * driver (gw_ldscore.py:1929-1956): with C (N x p) and R (p x N, both
 * column-major) and optional resvar_gram (p x p row-major), inv_out[j] =
 * 1/sqrt(max(eps, (||x_j||^2 + q - 2h)/(N - p - 1))) with h = ||R x_j||^2 and
 * q = (R x_j)^T gram (R x_j) (or h) (compute_inv_resvar_from_geno_block,
 * :3220-3333).  project_right != 0 with C and R projects the block's
 * genotypes, X <- (I - C R) X, before the products (:1633-1650; an error
 * together with inv_out, as in the reference).
 * ------------------------------------------------------------------- */
int lds_phase1_compute_Xz_bed_chunk_f32(
    const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, const float* annot_blk,
    int64_t annot_rows, int64_t K, const float* inv_right, int v_start, int v_count,
    int kmax_hint, int rand_dist, int has_seed, uint64_t seed, float* Xz2d_chunk,
    int64_t xz_rows, int64_t xz_cols, uint8_t* bin_init_mask, int impute_mode,
    int has_impute_seed, uint64_t impute_seed, float* inv_out, double resvar_eps,
    const float* C, const float* R, int64_t p, const float* resvar_gram, int project_right);
int lds_phase1_compute_Xz_bed_chunk_f64(
    const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, const double* annot_blk,
    int64_t annot_rows, int64_t K, const double* inv_right, int v_start, int v_count,
    int kmax_hint, int rand_dist, int has_seed, uint64_t seed, double* Xz2d_chunk,
    int64_t xz_rows, int64_t xz_cols, uint8_t* bin_init_mask, int impute_mode,
    int has_impute_seed, uint64_t impute_seed, double* inv_out, double resvar_eps,
    const double* C, const double* R, int64_t p, const double* resvar_gram, int project_right);

/* ---------------------------------------------------------------------
 * Phase 2: Work = X_blk^T Xz2d; meansq_accum[blk_start+j, k] +=
 * max(0, sum_{c in bin k} Work_jc^2 * inv_j^2 / (N_denom-1)^2) with the
 * reference's non-finite / extreme-update guards, and the optional
 * fourth-moment sums.  Replaces gwldcore.phase2_accum_XtXz_bed
 * (gwldcore.cpp:3759-3770, implementation :2329-2600).  Xz2d is N x Q
 * column-major with Q = K*tile_nvecs; meansq_accum is M x K row-major;
 * mc_aggregate_sumsq (K doubles) and mc_per_snp_sumsq (M x K doubles) may be
 * NULL.  With C and R (p > 0) the products use the projected genotypes,
 * Work = ((I - C R) X)^T Xz2d (:2376-2390).
 * ------------------------------------------------------------------- */
int lds_phase2_accum_XtXz_bed_f32(
    const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, const float* inv_left, int64_t L,
    int tile_nvecs, const float* Xz2d, int64_t xz_rows, int64_t xz_cols, float* meansq_accum,
    int64_t M_rows, int64_t K, int N_denom, int impute_mode, int has_impute_seed,
    uint64_t impute_seed, double* mc_aggregate_sumsq, double* mc_per_snp_sumsq, const float* C,
    const float* R, int64_t p);
int lds_phase2_accum_XtXz_bed_f64(
    const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, const double* inv_left, int64_t L,
    int tile_nvecs, const double* Xz2d, int64_t xz_rows, int64_t xz_cols,
    double* meansq_accum, int64_t M_rows, int64_t K, int N_denom, int impute_mode,
    int has_impute_seed, uint64_t impute_seed, double* mc_aggregate_sumsq,
    double* mc_per_snp_sumsq, const double* C,
    const double* R, int64_t p);

/* ---------------------------------------------------------------------
 * Residual variances: inv[j] = 1/sqrt(max(eps, ||x_j||^2 / (N-1))) for all
 * nsnps SNPs, or with covariates (C N x p, R p x N column-major)
 * inv[j] = 1/sqrt(max(eps, ||(I - C R) x_j||^2 / (N - p - 1))); snp_var_out
 * (may be NULL) receives min(1, ||(I - C R) x_j||^2 / ||x_j||^2).  Replaces
 * gwldcore.precompute_residual_variances_bed (gwldcore.cpp:3748-3757,
 * implementation :3335-3566).  compute_mu22 != 0 also writes mu22_out
 * (B x B row-major): with S = sum_j (x'_j o x'_j) annot_all[j, k] inv_j^2
 * (x' the projected standardized genotypes; annot_all nsnps x B row-major),
 * mu22[a][b] = (S^T S)[a][b] / (N Msum_a Msum_b), 0 where the denominator is
 * 0 or the value not finite (:3421-3563).
 * ------------------------------------------------------------------- */
int lds_precompute_residual_variances_bed_f32(
    const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, double eps, int impute_mode,
    int has_impute_seed, uint64_t impute_seed, float* inv_out, const float* C, const float* R,
    int64_t p, double* snp_var_out, int compute_mu22, const float* annot_all,
    int64_t annot_rows, int64_t B, double* mu22_out);
int lds_precompute_residual_variances_bed_f64(
    const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
    const int64_t* row_sel, int64_t n_row_sel, int ddof, double eps, int impute_mode,
    int has_impute_seed, uint64_t impute_seed, double* inv_out, const double* C,
    const double* R, int64_t p, double* snp_var_out, int compute_mu22, const double* annot_all,
    int64_t annot_rows, int64_t B, double* mu22_out);

/* ---------------------------------------------------------------------
 * Whole genome-wide LD-score estimate in one call (all V-tiles, all SNP
 * blocks, residual variances, phase 1, untouched-bin zeroing, phase 2,
 * division by the probe count and the M_k/N_denom null), i.e. the native
 * work of GenomewideLDScore._compute_ldscore (gw_ldscore.py:1753-2222)
 * without covariates.  The genotype image stays on the device for the whole
 * call; probes follow the reference's per-block mt19937_64 streams, so the
 * result equals the reference's on the same seed, blocks and V-tiles.
 *
 * bed_rows: SNP-major packed BED rows (no 3-byte header), M rows of
 *   bed_row_bytes >= ceil(n_total/4) bytes, host memory.
 * annot: M x K row-major float64.  ldscore / meansq_accum: M x K float64
 *   outputs.  inv_out (M, may be NULL).  mc_* may be NULL.
 * as_float != 0 reproduces the float32 path's inputs (float probes and
 *   float-rounded residual variances).
 * ------------------------------------------------------------------- */
int lds_gw_ldscore(
    const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total, int64_t M,
    const int64_t* row_sel, int64_t n_row_sel, const double* annot, int64_t K,
    int nvecs, int step_size, int vtile, uint64_t seed, int rand_dist, int ddof,
    int impute_mode, uint64_t impute_seed, double resvar_eps, int as_float,
    double* ldscore, double* meansq_accum, double* inv_out,
    double* mc_aggregate_sumsq, double* mc_per_snp_sumsq);

/* Same as lds_gw_ldscore, reading the fileset `bed_prefix`.bed/.bim/.fam. */
int lds_gw_ldscore_bed(
    const char* bed_prefix, const char* fam_path, const int64_t* row_sel,
    int64_t n_row_sel, const double* annot, int64_t K, int nvecs, int step_size, int vtile,
    uint64_t seed, int rand_dist, int ddof, int impute_mode, uint64_t impute_seed,
    double resvar_eps, int as_float, double* ldscore, double* meansq_accum,
    double* inv_out, double* mc_aggregate_sumsq, double* mc_per_snp_sumsq);

/* ---------------------------------------------------------------------
 * Resident form of lds_gw_ldscore for repeated runs and timing.
 *   lds_geno_create: upload + repack + per-SNP statistics (+ HWE imputation)
 *     of a BED image into device memory; returns a handle.
 *   lds_gw_plan_create: residual variances, CSR lists, probe streams and all
 *     other kernel inputs of one estimate, uploaded; returns a plan.
 *   lds_gw_plan_execute: enqueue the estimate's kernels (phase 1 weights,
 *     phase 1, sketch digits, phase 2) on the library stream; asynchronous.
 *   lds_gw_plan_results: wait, then copy out and finalize like lds_gw_ldscore.
 *   lds_gw_plan_kernel_ms: CUDA-event time per kernel kind of the last
 *     execute: [weights, phase 1, sketch digits, phase 2] in ms (plans with at
 *     most 3 V-tiles).
 * No reference counterpart as single calls: together they perform the
 * native work of gw_ldscore.py:1753-2222 like lds_gw_ldscore.
 * ------------------------------------------------------------------- */
int lds_set_stream(void* cuda_stream); /* NULL restores the library's own stream */
int lds_geno_create(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total, int64_t M,
                    const int64_t* row_sel, int64_t n_row_sel, int impute_mode,
                    uint64_t impute_seed, int ddof, int64_t* handle_out);
/* Resident image of the library's seeded synthetic genotypes (the bytes of
 * lds_synth_bed) generated on the device, with no host copy: t0/t1 are the
 * per-SNP HWE thresholds (M each); no counterpart in the reference. */
int lds_geno_create_synthetic(int64_t n_total, int64_t M, uint64_t seed, const int64_t* t0,
                              const int64_t* t1, int missing, int impute_mode,
                              uint64_t impute_seed, int ddof, int64_t* handle_out);
int lds_geno_destroy(int64_t handle);
int lds_gw_plan_create(int64_t geno, const double* annot, int64_t K, int nvecs, int step_size,
                       int vtile, uint64_t seed, int rand_dist, double resvar_eps, int as_float,
                       int with_mc, int64_t* plan_out);
int lds_gw_plan_execute(int64_t plan);
int lds_gw_plan_results(int64_t plan, double* ldscore, double* meansq_accum, double* inv_out,
                        double* mc_aggregate_sumsq, double* mc_per_snp_sumsq);
int lds_gw_plan_kernel_ms(int64_t plan, double* ms4);
int lds_gw_plan_destroy(int64_t plan);

/* ---------------------------------------------------------------------
 * SNP shards across GPUs (one process per GPU).  Phase 1 is a sum over SNP
 * blocks, so each rank holds a contiguous SNP shard as its own genotype
 * image, computes the partial sketch of its SNPs, and the ranks sum the
 * sketches (one all-reduce per V-tile); phase 2 is then independent per
 * shard.  The caller owns the exchange (e.g. an NCCL all-reduce on the
 * stream set with lds_set_stream).  No single reference counterpart: the
 * reference runs the same sum over SNP blocks in one process
 * (gw_ldscore.py:1934-2019 phase-1 loop, :2060-2160 phase-2 loop).
 *   lds_gw_plan_create_shard: lds_gw_plan_create for a genotype image that
 *     holds SNPs [snp_offset, snp_offset + M) of the fileset; snp_offset is
 *     a multiple of step_size, so the shard's blocks and their probe streams
 *     (keyed by the block's start in the fileset) are the unsharded ones.
 *     Mean imputation only (HWE draws are keyed by the fileset SNP index).
 *   lds_gw_plan_tiles: number of V-tiles, their probe counts (tile_sizes
 *     may be NULL) and the sketch's row count N_pad (may be NULL).
 *   lds_gw_plan_phase1: enqueue phase 1 of V-tile `tile` into the caller's
 *     device buffer d_sketch (N_pad x K*V FP64, column-major, column k*V+v;
 *     every element written; rows >= N are finite and ignored by phase 2).
 *     Tile 0 also zeroes the plan's accumulators.
 *   lds_gw_plan_phase2: enqueue phase 2 of V-tile `tile` from d_sketch (the
 *     all-reduced sketch) into the plan's accumulators.
 *   lds_gw_plan_set_bin_totals / lds_gw_plan_bin_totals: the per-bin
 *     annotation totals M_k used by lds_gw_plan_results' finalize (default:
 *     the shard's own; set them to the sum over shards).
 * ------------------------------------------------------------------- */
int lds_gw_plan_create_shard(int64_t geno, const double* annot, int64_t K, int nvecs,
                             int step_size, int vtile, uint64_t seed, int rand_dist,
                             double resvar_eps, int as_float, int with_mc, int64_t snp_offset,
                             int64_t* plan_out);
int lds_gw_plan_tiles(int64_t plan, int* n_tiles, int* tile_sizes, int64_t* sketch_rows);
int lds_gw_plan_phase1(int64_t plan, int tile, double* d_sketch);
int lds_gw_plan_phase2(int64_t plan, int tile, const double* d_sketch);
int lds_gw_plan_set_bin_totals(int64_t plan, const double* Mk);
int lds_gw_plan_bin_totals(int64_t plan, double* Mk);

/* ---------------------------------------------------------------------
 * Windowed + partitioned LD scores (stochastic, probe based).  Windows are a
 * contiguous partition of the SNPs: window w = [window_starts[w],
 * window_starts[w+1]), window_starts[0] = 0, window_starts[n_windows] = M.
 * For SNP j in window w and bin k the estimate is the genome-wide estimator
 * restricted to window w: sum over probes of (x_j^T X_w D_k z)^2 scaled as in
 * phase 2, divided by nvecs, minus M_{w,k}/(N - ddof).  Window w draws its
 * own probes: root seed lds_window_seed(seed, w), SNP blocks of step_size
 * counted from the window start — so window w's scores equal lds_gw_ldscore
 * on the window's SNPs with that seed.  All windows run as batched phase-1
 * super-bins and a tile-table phase 2; the first execute captures the whole
 * estimate into one CUDA graph and later executes launch that graph.
 * batch_gb bounds the int8 sketch digits of one window batch (<= 0: 8 GB).
 * No single reference counterpart: the reference's windowed scores are
 * exact (winldcore.cpp:783-931); this is the probe estimator of
 * gw_ldscore.py:1753-2222 applied per window.
 * ------------------------------------------------------------------- */
int lds_win_plan_create(int64_t geno, const double* annot, int64_t K,
                        const int64_t* window_starts, int64_t n_windows, int nvecs,
                        int step_size, int vtile, uint64_t seed, int rand_dist, double resvar_eps,
                        int as_float, int with_mc, double batch_gb, int64_t* plan_out);
int lds_win_plan_execute(int64_t plan);
int lds_win_plan_results(int64_t plan, double* ldscore, double* meansq_accum, double* inv_out,
                         double* mc_per_snp_sumsq);
int lds_win_plan_kernel_ms(int64_t plan, double* ms4);
/* Per-window annotation totals M_{w,k} (n_windows x K row-major, summed in SNP
 * order within each window), the null the finalize subtracts as
 * M_{w,k} / (N - ddof); the windowed counterpart of lds_gw_plan_bin_totals. */
int lds_win_plan_bin_totals(int64_t plan, double* mkw_out);
/* Tiling of one windowed plan, set before its first execute (the autotuner's
 * knob; summit_b200/autotune.py chooses it, with the window batch size, by
 * timing):
 *   p1_sb_per_cta: phase-1 super-bins (window x bin) per CTA, i.e. how the
 *     super-bin work list is split across CTAs (0: default 8).
 * The LD scores do not depend on the tiling (bit for bit).  No reference
 * counterpart (it replaces the reference's CPU tiling environment knobs). */
int lds_win_plan_set_tiling(int64_t plan, int p1_sb_per_cta);
/* Phase-2 CTA order of a windowed plan, set before its first execute (the
 * autotuner's knob; no reference counterpart): window by window, chunks of
 * about bin_chunk bins (whole bin groups of lds_win_plan_set_p2_bins, at
 * least one), the window's 128-SNP tiles, the chunk's bin groups, so that the
 * CTAs that run together share a tile's packed codes and a (window, bin)
 * sketch in L2 (default 4; 0: grid order, bins slowest).  The scores do not
 * depend on it (bit for bit). */
int lds_win_plan_set_p2_order(int64_t plan, int bin_chunk);
/* Bins per phase-2 CTA of a windowed plan, set before its first execute (the
 * autotuner's knob; no reference counterpart).  A CTA walks its bins' sketch
 * columns in MMA groups of up to 256, a bin possibly straddling two groups;
 * 0 (default) takes the smallest count with the fewest groups per 128-SNP
 * tile (6 for K = 24 bins of 50 probes: 20 groups of 256 columns instead of
 * 24 of 208).  The scores do not depend on it (bit for bit). */
int lds_win_plan_set_p2_bins(int64_t plan, int bins_per_cta);
/* Exact integrity check of the phase-2 tensor-core products (the counterpart
 * of the reference's ABFT / Freivalds check of its GxE GEMMs,
 * gxeldcore.cpp:4674-4734, made exact because the products are integers).
 * With checks on (set before the plan's first execute), every estimate also
 * forms per SNP j two pairs of wrapping 64-bit checksums: lhs from the phase-2
 * epilogue, sum over (bin k, probe v) of h(k, v) times the exact products
 * G_j^T y~_kv and O_j^T y~_kv, and rhs = sum_i g_ij u(i), sum_i o_ij u(i) with
 * u(i) = sum h(k, v) y~_kv(i), recomputed on the CUDA cores from the sketch
 * digits and the packed codes (h odd, so any single wrong product shows).
 * lds_win_plan_check copies both (2 x M each, [2j] G and [2j+1] O; either
 * pointer may be NULL) and compares them on the host: mismatches = SNPs that
 * differ, first_snp the first (-1 if none), check_ms the check kernels' time
 * in the last estimate.  lds_check_vectors is that host comparison alone (for
 * checksums a caller copied or stored). */
/* Bounds-checked build (python -m summit_b200.build --checked, which writes
 * liblds_checked.so; no reference counterpart, it stands in for the
 * reference's sanitizer builds, CMakeLists.txt:476-515): the tensor-core
 * kernels check their tile, bin, sketch-column, member-row and output indices,
 * and a failed check records its code in a device error word and skips the
 * access instead of trapping.  lds_checked_build: 1 in that build, 0 otherwise.
 * lds_checked_errors: the first failed check's code since the last call (0:
 * none; always 0 in the ordinary build), then clears it. */
int lds_checked_build(void);
int lds_checked_errors(unsigned* code_out);
int lds_win_plan_set_checks(int64_t plan, int on);
/* The same checks on a genome-wide plan (lds_gw_plan_create; the tcgen05 path):
 * its rows form one window. */
int lds_gw_plan_set_checks(int64_t plan, int on);
int lds_gw_plan_check(int64_t plan, unsigned long long* lhs, unsigned long long* rhs,
                      int64_t* mismatches, int64_t* first_snp, double* check_ms);
int lds_win_plan_check(int64_t plan, unsigned long long* lhs, unsigned long long* rhs,
                       int64_t* mismatches, int64_t* first_snp, double* check_ms);
int lds_check_vectors(const unsigned long long* lhs, const unsigned long long* rhs, int64_t n_snps,
                      int64_t* mismatches, int64_t* first_snp);
int lds_win_plan_destroy(int64_t plan);

/* Windowed + partitioned LD scores in one call from host BED rows (the
 * one-call form of lds_geno_create + lds_win_plan_create/execute/results,
 * like lds_gw_ldscore for the genome-wide estimate; no single reference
 * counterpart, see lds_win_plan_create).  The upload is streamed: the windows
 * are cut into window-aligned chunks of about M / n_chunks SNPs (n_chunks <= 0:
 * 8; 1: one chunk, no overlap), the first two of them a quarter and a half of
 * that size, and chunk i+1's upload, repack, per-SNP statistics and plan
 * set-up run on a second stream while chunk i's estimate runs on the library
 * stream.  Chunk memory
 * comes from a library-private stream-ordered pool that keeps its
 * reservation between calls (lds_clear_device_cache releases it).
 * Window seeds are counted from the global window index and HWE imputation
 * seeds from the global SNP index, so the scores equal lds_win_plan_results
 * of one plan over the whole image (same seed, windows, V-tiles) bit for bit.
 * bed_rows: M rows of bed_row_bytes >= ceil(n_total/4) bytes (pinned host
 * memory uploads at full PCIe rate).  p1_sb_per_cta: the chunks' tiling as
 * in lds_win_plan_set_tiling (0: default).  ldscore: M x K;
 * meansq_accum (M x K) and inv_out (M) may be NULL.  Returns after all
 * outputs are written. */
int lds_win_ldscore(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total, int64_t M,
                    const int64_t* row_sel, int64_t n_row_sel, const double* annot, int64_t K,
                    const int64_t* window_starts, int64_t n_windows, int nvecs, int step_size,
                    int vtile, uint64_t seed, int rand_dist, int ddof, int impute_mode,
                    uint64_t impute_seed, double resvar_eps, int as_float, int n_chunks,
                    int p1_sb_per_cta, double* ldscore, double* meansq_accum, double* inv_out);

/* Control-variate outputs of a windowed plan (no counterpart in the reference;
 * they serve the learned control variate).  Call lds_win_plan_set_cv before the
 * plan's first execute.  split_tiles != 0 keeps two meansq slices, probes
 * [0, h) and [h, nvecs) with h = ceil(nvecs / 2) (independent probe sets, so
 * their spread estimates the Monte-Carlo noise);
 * band_D in {4, 8, 15} also computes, per (SNP j, bin k),
 *   mu[j K + k] = sum_{|i-j| <= D, same window} c_ji^2 annot_ik^2   (exact) and
 *   C[t][j K + k] = sum_v (sum_{same i} c_ji annot_ik z_iv)^2   (probes of slice t),
 * c_ji = (x_j . x_i) sqrt(left scale_j) from lds_nn_band's exact products, so
 * that meansq - C + V mu is an unbiased near-field control-variate estimate
 * of meansq.  band_D = 0 disables it.  annot: M x K row-major (as at create). */
int lds_win_plan_set_cv(int64_t plan, const double* annot, int split_tiles, int band_D);
/* Device address of the plan's copy of the annotation matrix (M x K
 * row-major float64, uploaded by lds_win_plan_set_cv; valid until the plan is
 * destroyed, read-only), so that callers on other streams need not upload it
 * again; the library stream is synchronized first. */
int lds_win_plan_cv_annot(int64_t plan, const double** d_annot);
/* Number of V-tiles and their probe counts (tile_sizes may be NULL). */
int lds_win_plan_tiles(int64_t plan, int* n_tiles, int* tile_sizes);
/* After execute: copy the outputs (host pointers, or device pointers when
 * device_ptrs != 0; any may be NULL).  meansq_tiles and C_tiles hold
 * n_out x M x K values (n_out = 2 with split_tiles, else 1); mu M x K;
 * xx M x (band_D+1).  Waits for the plan's work. */
int lds_win_plan_cv_outputs(int64_t plan, int device_ptrs, double* meansq_tiles,
                            double* C_tiles, double* mu, double* xx);
/* Device time (ms) of the control-variate kernels of the last execute. */
int lds_win_plan_cv_ms(int64_t plan, double* ms);
uint64_t lds_window_seed(uint64_t root, int64_t w);
/* One Rademacher probe block generated on the device (L x V column-major, host
 * output): the std::mt19937_64 stream of make_seed(root, blk_start, v_start)
 * (gwldcore.cpp:452-458, :1702-1706) that the plans use for Rademacher probes. */
int lds_debug_rademacher_block(uint64_t root, int blk_start, int v_start, int L, int V,
                               double* out);

/* Device timing of the last lds_gw_ldscore call (milliseconds, CUDA events
 * on the library stream): [0] upload+prepare, [1] phase 1 total, [2] phase 2
 * total, [3] whole call.  After lds_win_ldscore: host wall-clock milliseconds
 * from its start to [0] the first chunk's estimate enqueued, [1] every
 * chunk's estimate enqueued, [2] every result copied out, [3] the chunks'
 * device buffers released (the whole call). */
int lds_last_timings(double* ms_out, int n);

/* Verification entry: exact int64 products G^T y and O^T y of the int8
 * columns y (n x Q, column-major) with the genotype rows of `bed_rows`
 * (L SNP rows of bed_row_bytes bytes, n samples), computed by the same int8
 * tensor-core phase-2 kernel as the LD-score path (one digit).  out_g/out_o:
 * L x Q row-major.  No reference counterpart: it exposes the exact-integer
 * core of the phase-2 product (gwldcore.cpp:2490 Geno^T.Xz) for testing. */
int lds_debug_xt_products(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n, int64_t L,
                          const int8_t* y, int64_t Q, int64_t* out_g, int64_t* out_o);

/* Same check through the tcgen05 phase-2 kernel: y is n x (4*V) int8,
 * column 4 v + t = digit t of probe v; out_g/out_o (L x V row-major) receive
 * the exact digit recombination ((d0*128 + d1)*128 + d2)*128 + d3 of the
 * per-digit products.  No reference counterpart (test entry). */
int lds_debug_xt_products_umma(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n,
                               int64_t L, const int8_t* y, int64_t V, int64_t* out_g,
                               int64_t* out_o);

/* Phase-2 kernel selection: 1 = tcgen05 (default), 0 = mma.sync.  Applies to
 * plans created afterwards.  No reference counterpart. */
int lds_set_p2_kernel(int impl);

/* Synthetic genotype image generated on the device with the integer-exact
 * generator (identical bytes to the numpy generator in bedfile.py):
 * writes M rows of ceil(n/4) bytes to host memory `out`.  t0/t1 are the
 * per-SNP integer latent thresholds. */
int lds_synth_bed(int64_t n, int64_t M, uint64_t seed, const int64_t* t0, const int64_t* t1,
                  int missing, uint8_t* out);

/* ---------------------------------------------------------------------
 * Exact products of each SNP with its D nearest right-hand neighbours on a
 * resident genotype image (lds_geno_create):
 *   xx_out[j*(D+1) + d] = x_j . x_{j+d}   (0 when j+d >= M),
 * x_ij = s_j (g_ij - mu_j) o_ij with the image's imputation, mean and sd (the
 * standardization of the stochastic estimators).  r^2 to a neighbour is
 * xx[j][d]^2 / (xx[j][0] xx[j+d][0]).  counts_out (may be NULL) receives the
 * exact integer sums GG, GO, OG, OO per (j, d), 4 int32 each.  These are the
 * near-diagonal entries of X^T X that the exact windowed LD scores
 * (compute_windowed_ld_chr_impl, winldcore.cpp:783, via syrk panels) sum in
 * full; here they feed the control variate.  0 <= D <= LDS_NN_BAND_MAX.
 * Synchronous.
 * ------------------------------------------------------------------- */
#define LDS_NN_BAND_MAX 15
/* Per-SNP mean (2 x allele frequency) and inverse sd of a resident image, as
 * used by its standardization (M values each; either pointer may be NULL). */
int lds_geno_stats(int64_t geno, double* mean_out, double* sdinv_out);
int lds_nn_band(int64_t geno, int D, double* xx_out, int32_t* counts_out);

/* ---------------------------------------------------------------------
 * Further gwldcore entry points (gwldcore.cpp:3656-3829), float and double:
 *
 * lds_phase1_compute_Xz_bed_chunk_rowmajor_*  (:3703-3718, impl :1925-2130):
 *   as the column-major phase 1, but Xz2d_chunk is N x K*v_count row-major and
 *   always accumulates (no bin_init_mask).
 * lds_phase2_accum_XtXz_bed_mailman_* (:3785-3794, impl :2651-2917) and
 *   lds_phase2_accum_XtXz_bed_mailman_rowmajor_* (:3796-3805, impl :2919-3119):
 *   phase 2 on HWE-completed genotypes (the Mailman path's imputation); the
 *   row-major form takes Xz2d row-major and the sketch's column sums sum_Xz
 *   (n_sum = Q), which are recomputed exactly on the device.
 * lds_compute_col_sums_rowmajor_* (:3720, impl :3121-3132): FP64 column sums
 *   of a row-major N x Q sketch (same summation order as the reference).
 * lds_project_rowmajor_inplace_and_col_sums_* (:3722-3725) and
 *   lds_project_colmajor_inplace_* (:3726-3729): X <- (I - C R) X with C N x p
 *   and R p x N column-major (no-op when either is NULL or p = 0); the
 *   row-major form also returns the column sums.
 * lds_standardize_dosage_inplace_* (:3664-3669, impl :1511-1580): per
 *   column (x - mean) / sd over calls in [0, 2] (ddof), missing and invalid
 *   calls set to 0; missing_out receives the count of missing calls;
 *   out-of-range non-missing calls are an error (after the update, as in the
 *   reference).
 * ------------------------------------------------------------------- */
#define LDS_P1R_ARGS(T)                                                                       \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                 \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *annot_blk,              \
        int64_t annot_rows, int64_t K, const T *inv_right, int v_start, int v_count,          \
        int kmax_hint, int rand_dist, int has_seed, uint64_t seed, T *Xz2d_chunk,              \
        int64_t xz_rows, int64_t xz_cols, int impute_mode, int has_impute_seed,               \
        uint64_t impute_seed, T *inv_out, double resvar_eps, const T *C, const T *R,          \
        int64_t p, const T *resvar_gram
int lds_phase1_compute_Xz_bed_chunk_rowmajor_f32(LDS_P1R_ARGS(float));
int lds_phase1_compute_Xz_bed_chunk_rowmajor_f64(LDS_P1R_ARGS(double));
#define LDS_P2M_ARGS(T)                                                                       \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                 \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,    \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,     \
        int64_t M_rows, int64_t K, int N_denom, int has_impute_seed, uint64_t impute_seed,    \
        double *mc_aggregate_sumsq, double *mc_per_snp_sumsq, const T *C, const T *R, int64_t p
int lds_phase2_accum_XtXz_bed_mailman_f32(LDS_P2M_ARGS(float));
int lds_phase2_accum_XtXz_bed_mailman_f64(LDS_P2M_ARGS(double));
#define LDS_P2MR_ARGS(T)                                                                      \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                 \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,    \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,     \
        int64_t M_rows, int64_t K, const double *sum_Xz, int64_t n_sum, int N_denom,          \
        int has_impute_seed, uint64_t impute_seed, double *mc_aggregate_sumsq,                \
        double *mc_per_snp_sumsq
int lds_phase2_accum_XtXz_bed_mailman_rowmajor_f32(LDS_P2MR_ARGS(float));
int lds_phase2_accum_XtXz_bed_mailman_rowmajor_f64(LDS_P2MR_ARGS(double));
int lds_compute_col_sums_rowmajor_f32(const float* X, int64_t N, int64_t Q, double* out);
int lds_compute_col_sums_rowmajor_f64(const double* X, int64_t N, int64_t Q, double* out);
int lds_project_rowmajor_inplace_and_col_sums_f32(float* X, int64_t N, int64_t Q, const float* C,
                                                  const float* R, int64_t p, double* sums);
int lds_project_rowmajor_inplace_and_col_sums_f64(double* X, int64_t N, int64_t Q,
                                                  const double* C, const double* R, int64_t p,
                                                  double* sums);
int lds_project_colmajor_inplace_f32(float* X, int64_t N, int64_t Q, const float* C,
                                     const float* R, int64_t p);
int lds_project_colmajor_inplace_f64(double* X, int64_t N, int64_t Q, const double* C,
                                     const double* R, int64_t p);
int lds_standardize_dosage_inplace_f32(float* G, int64_t N, int64_t L, int ddof,
                                       double missing_value, int64_t* missing_out);
int lds_standardize_dosage_inplace_f64(double* G, int64_t N, int64_t L, int ddof,
                                       double missing_value, int64_t* missing_out);

/* ---------------------------------------------------------------------
 * Dense genotype blocks (PGEN dosages and other callers that standardize
 * themselves): geno is N x L column-major, already standardized.
 * lds_phase1_compute_Xz_geno_chunk_* replaces phase1_compute_Xz_geno_chunk
 * (gwldcore.cpp:3690-3701, impl :1896-1923): the phase-1 update of the BED
 * form with the block's SNPs blk_start.. (probe streams keyed by blk_start),
 * inv_out / C / R / resvar_gram as there (no project_right).
 * lds_phase2_accum_XtXz_geno_* replaces phase2_accum_XtXz_geno
 * (:3772-3783, impl :2624-2649); with C and R the block is projected in
 * place, geno <- (I - C R) geno, as the reference does to the caller's array.
 * The FP64 products run on the device (dense, no digit split).
 * ------------------------------------------------------------------- */
#define LDS_P1G_ARGS(T)                                                                       \
    const T *geno, int64_t N, int64_t L, int blk_start, const T *annot_blk, int64_t annot_rows, \
        int64_t K, const T *inv_right, int v_start, int v_count, int kmax_hint, int rand_dist, \
        int has_seed, uint64_t seed, T *Xz2d_chunk, int64_t xz_rows, int64_t xz_cols,           \
        uint8_t *bin_init_mask, const T *C, const T *R, int64_t p, const T *resvar_gram,        \
        T *inv_out, double resvar_eps
int lds_phase1_compute_Xz_geno_chunk_f32(LDS_P1G_ARGS(float));
int lds_phase1_compute_Xz_geno_chunk_f64(LDS_P1G_ARGS(double));
#define LDS_P2G_ARGS(T)                                                                       \
    T *geno, int64_t N, int64_t L, int blk_start, const T *inv_left, int64_t L_in,             \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,      \
        int64_t M_rows, int64_t K, const T *C, const T *R, int64_t p, int N_denom,             \
        double *mc_aggregate_sumsq, double *mc_per_snp_sumsq
int lds_phase2_accum_XtXz_geno_f32(LDS_P2G_ARGS(float));
int lds_phase2_accum_XtXz_geno_f64(LDS_P2G_ARGS(double));

/* Legacy direct phase 2, replaces phase2_compute_XtXz_bed (gwldcore.cpp:
 * 3731-3740, impl :2132-2327): meansq += max(0, sum_c Work^2 inv^2 /
 * (nvecs (N_denom - 1)^2)) with the guards, Xz2d N x K*nvecs. */
#define LDS_P2L_ARGS(T)                                                                       \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                 \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,    \
        int nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq, int64_t M_rows, \
        int64_t K, const T *C, const T *R, int64_t p, int N_denom, int impute_mode,           \
        int has_impute_seed, uint64_t impute_seed
int lds_phase2_compute_XtXz_bed_f32(LDS_P2L_ARGS(float));
int lds_phase2_compute_XtXz_bed_f64(LDS_P2L_ARGS(double));

/* GRM panel products, replaces apply_grm_bed_panel / _mailman
 * (gwldcore.cpp:3812-3828, impl :1134-1497): panel_out = P X D X^T P panel_in
 * over SNPs [0, nsnps), D = diag(inv_all_j^2 / nsnps) (0 where not finite or
 * <= 0), P = I - C R when C and R are given; panels N x Q column-major.  The
 * Mailman form uses HWE-completed genotypes (impute_seed).  X^T V runs on the
 * tensor-core phase-2 kernel's exact raw-product mode, X (D coef) on the
 * phase-1 kernel. */
#define LDS_GRM_ARGS(T)                                                                       \
    const char *bed_prefix, const char *fam_path, int nsnps, int step_size,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_all, int64_t n_inv, \
        const T *panel_in, T *panel_out, int64_t rows, int64_t Q, const T *C, const T *R,     \
        int64_t p, int impute_mode, int has_impute_seed, uint64_t impute_seed
int lds_apply_grm_bed_panel_f32(LDS_GRM_ARGS(float));
int lds_apply_grm_bed_panel_f64(LDS_GRM_ARGS(double));
#define LDS_GRMM_ARGS(T)                                                                      \
    const char *bed_prefix, const char *fam_path, int nsnps, int step_size,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_all, int64_t n_inv, \
        const T *panel_in, T *panel_out, int64_t rows, int64_t Q, const T *C, const T *R,     \
        int64_t p, int has_impute_seed, uint64_t impute_seed
int lds_apply_grm_bed_panel_mailman_f32(LDS_GRMM_ARGS(float));
int lds_apply_grm_bed_panel_mailman_f64(LDS_GRMM_ARGS(double));

/* Block corrections of binary annotations, replaces
 * compute_block_corrections_binary (gwldcore.cpp:3807-3810, impl :3569-3627):
 * M_a = #{i: annot_ia != 0}, S_ab = sum_{i: annot_ia != 0} meansq_raw[i, b],
 * R2 = S / (M_a M_b), rho2 = (d^2 R2 - N mu22) / (N (N - 1)),
 * bias = S - M_a M_b rho2, delta = mu22 - (1 + 2 rho2) (0 where M_a, M_b or
 * S is 0); outputs B x B row-major.  annot_all is float32 or float64. */
#define LDS_BCB_ARGS(T)                                                                       \
    const double *meansq_raw, int64_t M, int64_t B, const double *mu22, const T *annot_all,   \
        int N, double d, double *R2, double *rho2, double *bias, double *delta
int lds_compute_block_corrections_binary_f32(LDS_BCB_ARGS(float));
int lds_compute_block_corrections_binary_f64(LDS_BCB_ARGS(double));

/* ---------------------------------------------------------------------
 * Exact windowed LD scores (tcgen05 int8 Gram products, FP64 epilogue).
 *
 * lds_compute_windowed_ld_chr replaces winldcore.compute_windowed_ld_chr
 * (winldcore.cpp:972-987, implementation :783-931): for SNPs j in
 * [chr_start, chr_end) of the BED fileset,
 *   out[j, b] = sum_{i : |bp_i - bp_j| <= 1000 ld_wind_kb} r~2_ij annot_chr[i, b]
 * with r the correlation of the mean-imputed (restandardized) or HWE-completed
 * genotypes over the selected samples and r~2 = r^2 - (1 - r^2)/(N - 2).
 * annot_chr and out are m x K column-major (m = chr_end - chr_start); bp has m
 * sorted positions.  Same argument checks and messages as the reference.
 * chunk_size must be > 0 but, like panel_cols and cache_mb (CPU tiling knobs),
 * does not change the result.  Covariate projection (C, R non-NULL with p > 0)
 * is rejected with LDS_ERR_ARG.
 *
 * lds_geno_window_ld is the same computation on a resident image with an
 * explicit partner interval per SNP: for j in [row0, row1),
 *   out[(j-row0)*K + b] = sum_{i in [lo[j-row0], hi[j-row0])} f(r_ij) annot[(i-row0)*K + b]
 * (row-major), f = r^2 when corr_dim <= 0 (the expectation of the stochastic
 * windowed estimator's meansq / B), else r^2 - (1 - r^2)/(corr_dim - 1).
 * Both are synchronous and deterministic.
 *
 * lds_compute_maf_bed replaces winldcore.compute_maf_bed (winldcore.cpp:988-993,
 * compute_maf_block genotype.cpp:1634): maf_out[j] for the first nsnps SNPs.
 * ------------------------------------------------------------------- */
int lds_compute_windowed_ld_chr(const char* bed_prefix, const char* fam_path, int chr_start,
                                int chr_end, const int64_t* bp, const double* annot_chr, int64_t K,
                                double ld_wind_kb, int chunk_size, const int64_t* row_sel,
                                int64_t n_row_sel, const double* C, const double* R, int64_t p,
                                int impute_mode, int has_impute_seed, uint64_t impute_seed,
                                int panel_cols, int cache_mb, double* out);
int lds_geno_window_ld(int64_t geno, int64_t row0, int64_t row1, const int64_t* lo,
                       const int64_t* hi, const double* annot, int64_t K, double corr_dim,
                       double* out);
int lds_compute_maf_bed(const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
                        const int64_t* row_sel, int64_t n_row_sel, double* maf_out);

/* ---------------------------------------------------------------------
 * SUMMIT-GxE multi-environment products on a resident genotype image
 * (replacing gxeldcore.MultiEnvironmentKernel, gxeldcore.cpp:10281-12557,
 * bindings :16420-16474).  N = samples of the image, E environments, K
 * annotation bins, B probes, T environments in a tile starting at env_start.
 * Arrays are column-major unless stated; accumulators are (E * total_variants)
 * x K row-major.  With device_ptrs = 0 every array argument is host memory
 * (copied per call); with 1 every array is a device pointer.
 *
 * lds_gxe_create: the kernel's constructor inputs (environments N x E, common
 *   basis N x r, directions N x E, feature basis N x F with power_indices /
 *   power_offsets (4E+1) / ranks (E)) — the power-0 range of environment e
 *   names its fixed-effect basis, on which projection leakage is measured.
 * lds_gxe_source_block (source_block, :11008-11240): target (N x T 2 K B)
 *   += X_[j0,j1) [sqrt(a) z s_x] (additive halves) and
 *   phi_e o X_[j0,j1) [sqrt(a) z s_w] (interaction halves); probes L x B,
 *   annotation L x K (square roots if annotation_is_sqrt), scales L x T.
 * lds_gxe_project_sources (project_sources, :11583-11729): in place; leakages
 *   receives one value per environment of the tile; leakage > 1e-9 is an error.
 * lds_gxe_pair_create (prepare_protected_row_weighted_pair, :9808): seals
 *   [right, w o right] (right N x C, row_weights N x G, column c weighted by
 *   w[:, c / (C / G)]) on the device.
 * lds_gxe_target_score_block (target_score_block, :11731-11936): out =
 *   X_[j0,j1)^T [S, w o S]; accumulates sum_b (s out)^2 / (N - rank_e)^2.
 * lds_gxe_normalize_scores (normalize_scores, :12490-12557): divides by B.
 * lds_philox_rademacher (numpy_philox_rademacher_block, :10070-10113): out
 *   rows x P of +-1 from NumPy Philox keys (P x 2 uint64), bit-identical to
 *   Generator(Philox).integers(0, 2, dtype=int8) * 2 - 1.
 * ------------------------------------------------------------------- */
int lds_gxe_create(int64_t geno, int64_t E, const double* environments, int64_t r,
                   const double* common_basis, const double* directions, int64_t F,
                   const double* feature_basis, const int64_t* power_indices,
                   const int64_t* power_offsets, const int32_t* ranks, int annotation_bins,
                   int64_t* handle_out);
/* Dense-block form, the reference binding's own argument: a context for N
 * samples whose source_block / target_score_block take the N x L column-major
 * FP64 standardized genotype block the reference's driver passes
 * (gxe_multi.py:3066-3230 -> gxeldcore.cpp:16420-16474) instead of an image
 * block; the products run as FP64 GEMMs on the device.  The other calls
 * (project_sources, pair_create, normalize_scores) take either context. */
int lds_gxe_create_dense(int64_t N, int64_t E, const double* environments, int64_t r,
                         const double* common_basis, const double* directions, int64_t F,
                         const double* feature_basis, const int64_t* power_indices,
                         const int64_t* power_offsets, const int32_t* ranks, int annotation_bins,
                         int64_t* handle_out);
int lds_gxe_source_block_dense(int64_t gxe, const double* genotype, int64_t L,
                               const double* probes, int64_t B, const double* annotation,
                               int annotation_is_sqrt, const double* scale_x,
                               const double* scale_w, int64_t T, int environment_start,
                               double* target, int device_ptrs);
int lds_gxe_target_score_block_dense(int64_t gxe, const double* genotype, int64_t L, int64_t pair,
                                     const double* scale_x, const double* scale_w, int64_t T,
                                     double* accum_xx, double* accum_xw, double* accum_wx,
                                     double* accum_ww, int64_t block_start,
                                     int64_t total_variants, int probe_count,
                                     int environment_start, int device_ptrs);
int lds_gxe_destroy(int64_t gxe);
/* Generalized per-variant GxE two-pass estimator (generalized_gxe_pass1.py
 * GeneralizedGxEPass1Executor, generalized_gxe_pass2.py
 * GeneralizedGxEPass2Executor), on a resident image (lds_geno_create) whose
 * standardized genotypes x_ij = s_j (g_ij - mu_j), 0 on a missing call, are
 * the decoded blocks of the reference's genotype operator.  Host pointers.
 * lds_geno_source_product: out (N x K*B column-major, column k*B + b) =
 *   sum_{j in [j0, j1)} x_j sqrt(a_jk) Z[j, b] (the pass-1 base sources);
 *   annot (L x K row-major) NULL means one unit-weight bin (K ignored).
 *   Z is L x B column-major.
 * lds_geno_target_product: out (L x cols column-major) = X_[j0,j1)^T Y, Y
 *   N x cols column-major (the pass-2 cross sketches).
 * lds_global_variant_probes: out (L x B column-major) = the reference's
 *   global_probe_sign (generalized_gxe_variant.py:80-103) for variants
 *   v0 .. v0+L-1 and probes p0 .. p0+B-1, namespace_key its FNV-1a key.
 * lds_generalized_component_diagonal: numerator (K*P x N row-major, component
 *   k*P + p, P = Q(Q+1)/2 pairs diagonal first) += sum_j a_jk kf_p f_q f_r
 *   with f_q(i, j) = phi_q(i) x_ij - sum_r F(i, r) coef[j, q, r] (the pass-2
 *   component-kernel diagonals, generalized_gxe_pass2.py:528-562); basis
 *   N x Q and fixed N x R column-major, coef L x Q x R row-major (NULL when
 *   R = 0); Q <= 6, R <= 16. */
int lds_geno_source_product(int64_t geno, int64_t j0, int64_t j1, const double* annot, int64_t K,
                            const double* Z, int64_t B, double* out);
int lds_geno_target_product(int64_t geno, int64_t j0, int64_t j1, const double* Y, int64_t cols,
                            double* out);
int lds_global_variant_probes(uint64_t root_seed, uint64_t namespace_key, int64_t v0, int64_t L,
                              int64_t p0, int64_t B, double* out);
/* lds_generalized_pass2: the per-variant pass-2 scores of all M variants in
 * blocks of variant_block rows.  rhs (N x K*B*F column-major, column
 * (k*B + b)*F + f: phi_t o contextual source s of annotation k, probe b, for
 * family f = (t, s)) is uploaded and quantized once; per block the phase-2
 * tensor-core kernel forms the exact products, and per variant j
 *   directional[j][tp][k*P + sp] = (1/B) sum over the orientation terms
 *   t in [term_off[tp*P + sp], term_off[tp*P + sp + 1]) of
 *   sum_b cross_{term_f1[t]} cross_{term_f2[t]},  cross = X^T rhs / residual_rank,
 * (directional: M x P x K*P, host) and directed (K*P x K*P) = sum_j a_jk1
 * directional[j][p1][.] (annot M x K row-major).  K*B*F <= 25,600. */
int lds_generalized_pass2(int64_t geno, const double* rhs, int K, int B, int F, int P,
                          const int* term_off, const int* term_f1, const int* term_f2,
                          double residual_rank, const double* annot, int64_t variant_block,
                          double* directional, double* directed);
/* Pass 1's projection of the contextual sources off the fixed effects
 * (GeneralizedGxEPass1Executor, generalized_gxe_pass1.py:718-757): base holds
 * K*B rows of N samples ((K, B, N): base source of annotation k, probe b),
 * basis N x Q and fixed N x R row-major (R <= 16, R = 0: no projection).
 * contextual (K*Q*B rows of N: row (k*Q + q)*B + b) = w - fixed fixed^T w with
 * w = basis[:, q] o base[k, b], in FP64 on the device.  max_abs / max_rel get
 * the reference's leakage measures: the largest |fixed^T p| entry and, over
 * (k, q), ||fixed^T P||_F / max(1, ||P||_F). */
int lds_generalized_project(const double* base, const double* basis, const double* fixed, int K,
                            int Q, int B, int R, int64_t N, double* contextual, double* max_abs,
                            double* max_rel);
/* lds_generalized_pass2 with the right-hand side formed on the device from
 * the contextual sources: sources holds K*Q*B rows of N samples (row
 * (k*Q + s)*B + b: source s of annotation k, probe b; the (K, Q, B, N) array
 * of GeneralizedGxEPass1Executor's sources), basis is N x Q row-major, and
 * family f = (fam_t[f], fam_s[f]) gives column (k*B + b)*F + f =
 * basis[:, t] o sources[k, s][b].  Only the sources and the basis cross PCIe
 * (K*Q*B*N + N*Q doubles instead of K*B*F*N). */
int lds_generalized_pass2_sources(int64_t geno, const double* sources, int Q, const double* basis,
                                  const int* fam_t, const int* fam_s, int K, int B, int F, int P,
                                  const int* term_off, const int* term_f1, const int* term_f2,
                                  double residual_rank, const double* annot,
                                  int64_t variant_block, double* directional, double* directed);
int lds_generalized_component_diagonal(int64_t geno, int64_t j0, int64_t j1, const double* annot,
                                       int K, const double* basis, int Q, const double* fixed,
                                       int R, const double* coef, double* numerator);
/* Generalized per-SNP GxE packed products (GeneralizedGxELDScoreDirectContext::
 * packed_source_product / packed_target_product, generalized_gxe_variant.inc:
 * 1749-1988) on a mean-imputed resident image (lds_geno_create): with the
 * Mailman mean pack's scale inv_j = sqrt((N - ddof) / M2_j) (genotype.cpp:
 * 1115-1131) and x'_j = inv_j (g_j - mu_j) on observed calls, 0 on missing,
 *   source: out (N x cols) = -X' rhs,   rhs (j1-j0) x cols column-major;
 *   target: out ((j1-j0) x cols) = -X'^T rhs,   rhs N x cols column-major
 * (the reference's out = mu sum - raw over packed allele counts). */
int lds_generalized_source_product(int64_t geno, int64_t j0, int64_t j1, const double* rhs,
                                   int64_t cols, double* out);
int lds_generalized_target_product(int64_t geno, int64_t j0, int64_t j1, const double* rhs,
                                   int64_t cols, double* out);
int lds_gxe_source_block(int64_t gxe, int64_t j0, int64_t j1, const double* probes, int64_t B,
                         const double* annotation, int annotation_is_sqrt, const double* scale_x,
                         const double* scale_w, int64_t T, int environment_start, double* target,
                         int device_ptrs);
int lds_gxe_project_sources(int64_t gxe, double* panel, int64_t columns,
                            int columns_per_environment, int environment_start, double* leakages,
                            int device_ptrs);
int lds_gxe_pair_create(int64_t gxe, const double* right, int64_t columns,
                        const double* row_weights, int64_t groups, int device_ptrs,
                        int64_t* pair_out);
int lds_gxe_pair_destroy(int64_t pair);
int lds_gxe_target_score_block(int64_t gxe, int64_t j0, int64_t j1, int64_t pair,
                               const double* scale_x, const double* scale_w, int64_t T,
                               double* accum_xx, double* accum_xw, double* accum_wx,
                               double* accum_ww, int64_t block_start, int64_t total_variants,
                               int probe_count, int environment_start, int device_ptrs);
int lds_gxe_normalize_scores(double* accum_xx, double* accum_xw, double* accum_wx,
                             double* accum_ww, int64_t rows, int64_t K, int probe_count,
                             int device_ptrs);
/* Exact integrity check of the GxE target's tensor-core products (the
 * counterpart of the reference's ABFT / Freivalds check of its GxE GEMMs,
 * gxeldcore.cpp:4674-4734, made exact because the products are integers; the
 * reference re-checks flagged columns under a floating-point bound and fails
 * on a material error).  With checks on (contexts on a resident image only),
 * every lds_gxe_target_score_block call also forms, per SNP, the checksums
 * sum_{k,v} h(k, v) T(j, k, v) of its products in the kernel's epilogue and
 * sum_i g_ij u(i) from the packed codes on the CUDA cores (G and O planes,
 * mod 2^64, h an odd weight per (group, probe)), compares them on the host
 * and returns LDS_ERR_INTERNAL if any SNP disagrees (the accumulators then
 * hold that call's suspect products). */
int lds_gxe_set_checks(int64_t gxe, int on);
/* The last checked target call: its checksums (2 x rows each, [G, O] per
 * SNP; either pointer may be null), first SNP, row count, mismatching SNPs
 * and the first of them (-1 if none). */
int lds_gxe_last_check(int64_t gxe, unsigned long long* lhs, unsigned long long* rhs,
                       int64_t* first_row, int64_t* rows, int64_t* mismatches,
                       int64_t* first_snp);
int lds_philox_rademacher(const uint64_t* keys, int64_t probes, int64_t rows, double* out,
                          int device_ptrs);

/* ---------------------------------------------------------------------
 * SNP-block jackknife and normal-equation solves in FP64 on the device
 * (inference/jackknife.py:109-214, context/fit.py:435-525, replicate SE of
 * inference/gxe.py:2052-2057).
 *
 * lds_block_boundaries: contiguous jackknife blocks of M SNPs; mass == NULL
 *   gives equal-count blocks (_equal_count_block_boundaries), otherwise
 *   weighted blocks (_weighted_contiguous_block_boundaries, min_snps per block).
 * lds_sym_solve: nsys systems laid out as (K*K row-major matrix, K rhs);
 *   symmetrize, eigendecompose, keep |lambda| > max(100 eps scale,
 *   rtol max|lambda|), x = sum_kept v (v^T b)/(v^T A v); rank and ascending
 *   eigenvalues per system (either may be NULL).  Asymmetry above 2e-10 scale,
 *   non-finite input, or (require_full_rank) rank < K is an error.  K <= 96.
 * lds_jackknife_normal_equations: terms is M x (K*K + K) per-SNP contributions
 *   [vec(A_j), b_j]; blocks [starts[b], ends[b]); theta = solve(sum A, sum b),
 *   replicates[b] = delete-block-b solutions, se = sqrt((B-1)/B sum (r - mean)^2),
 *   cov the matching covariance (rank-revealing solves, rtol).
 * ------------------------------------------------------------------- */
int lds_block_boundaries(int64_t M, int B, const double* mass, int min_snps, int64_t* starts,
                         int64_t* ends);
int lds_sym_solve(const double* systems, int64_t nsys, int K, double rtol, int require_full_rank,
                  double* x, int* rank, double* eigenvalues, int device_ptrs);
/* lds_sym_solve_diag: the same solve with the diagnostics of
 * solve_context_normal_equations / _rank_diagnostics (context/fit.py:435-513):
 * per system x (K), rank, ascending eigenvalues (K), eigenvectors (K x K
 * row-major, column p for the p-th eigenvalue), residual S x - b (K; S the
 * symmetrized matrix), symmetry error max|A - A^T|, the retention tolerance,
 * and status bits (1 asymmetry above 2e-10 scale, 4 non-finite input) that
 * the caller turns into its errors.  Rank deficiency is reported, not an
 * error.  Host pointers (any output may be NULL); K <= 96. */
int lds_sym_solve_diag(const double* systems, int64_t nsys, int K, double rtol, double* x,
                       int* rank, double* eigenvalues, double* eigenvectors, double* residual,
                       double* symmetry_error, double* tolerance, int* status);
int lds_jackknife_normal_equations(const double* terms, int64_t M, int K, const int64_t* starts,
                                   const int64_t* ends, int64_t B, double rtol, double* theta,
                                   double* replicates, double* se, double* cov, int device_ptrs);

/* ---------------------------------------------------------------------
 * Surrogate network of the learned control variate (no counterpart in the
 * reference): in_dim -> 128 -> 128 -> 128 -> out_dim, GELU (erf form) after the
 * hidden layers, FP32 master parameters, BF16 weights and activations in the
 * products with FP32 accumulation.  Parameters are one FP32 array of
 * lds_mlp_param_count floats: W1 [128][in], b1 [128], W2 [128][128], b2,
 * W3 [128][128], b3, W4 [out][128], b4 [out] (row-major).  All pointers are
 * device pointers owned by the caller; x is n x in_dim, targets and outputs
 * n x out_dim (row-major FP32).  The loss is the mean over rows and outputs of
 * the squared error.  Calls are synchronous.
 * ------------------------------------------------------------------- */
#define LDS_MLP_MAX_IN 128
#define LDS_MLP_MAX_OUT 64
int64_t lds_mlp_param_count(int in_dim, int out_dim);
int lds_mlp_forward(const float* d_params, int in_dim, int out_dim, const float* d_x, int64_t n,
                    float* d_out);
/* d_grad (param_count floats) = gradient of the loss over all n rows; loss_out (host). */
int lds_mlp_loss_grad(const float* d_params, int in_dim, int out_dim, const float* d_x,
                      const float* d_t, int64_t n, float* d_grad, double* loss_out);
/* Adam (beta 0.9 / 0.999, eps 1e-8, rate lr) over shuffled mini-batches of
 * `batch` rows for `epochs` passes, in place on d_params; loss_per_epoch (host,
 * may be NULL) receives each epoch's mean mini-batch loss. */
int lds_mlp_train(float* d_params, int in_dim, int out_dim, const float* d_x, const float* d_t,
                  int64_t n, int epochs, int batch, float lr, uint64_t seed,
                  double* loss_per_epoch);

/* ---------------------------------------------------------------------
 * Phase 2 without any device allocation.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory during this step — work
 * captured into a CUDA graph (an allocation would break the capture),
 * programs whose device memory belongs to another framework's pool, and
 * services that forbid allocator calls after start-up.  The caller passes
 * device buffers it owns; the library's scratch (4-digit sketch split,
 * column scales, status words) is one fixed array of
 * LDS_NOALLOC_SCRATCH_BYTES held by every GPU that loads liblds.so until the
 * process exits.  Requires K * ceil16(4 V) * 4 row_bytes + 8 K V + ~1 KiB
 * <= LDS_NOALLOC_SCRATCH_BYTES; larger sizes are rejected with LDS_ERR_ARG.
 *
 *   d_codes: packed genotype rows in the library's device layout: row j at
 *     d_codes + j*row_bytes, row_bytes a multiple of 64 (N_pad = 4 row_bytes
 *     samples), sample i in bits 2(i%4) of byte i/4, samples >= n coded 01;
 *     16-byte aligned; rows_total rows addressable (rows_total >= j1).
 *   d_Y: sketch, N_pad x (K*V) column-major (column k*V + v), FP64.
 *   d_mean, d_sdinv, d_left_scale: per SNP row (index j), FP64.
 *   d_accum: (j1-j0) x K row-major FP64, += sum_v Work^2 * left_scale with
 *     the guards of lds_phase2_accum_XtXz_bed (SUMMIT_P2_EXTREME_LD_WARN,
 *     SUMMIT_P2_DROP_EXTREME); d_mc (may be NULL) += the fourth-moment sums.
 *   d_status (may be NULL): one caller-owned device word that receives the
 *     kernel's status (0 = ok; nonzero = a pipeline wait ran out and the
 *     accumulators are incomplete); d_guards (may be NULL): two device
 *     words that receive the numbers of non-finite and extreme updates
 *     dropped.  With d_status given the call is asynchronous on `stream`
 *     (cudaStream_t or NULL) and the words are written on that stream after
 *     the kernel.  With d_status NULL the call waits for its own work on
 *     `stream`, prints the guard warnings, and returns LDS_ERR_CUDA when the
 *     kernel aborted.
 * The first call on each device looks up the scratch array's address
 * (cudaGetSymbolAddress) and must come before any stream capture.  All
 * calls share the array and it keeps the last call's contents, so calls
 * that overlap on the GPU race; serialize them.
 * ------------------------------------------------------------------- */
#define LDS_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int lds_phase2_accum_device_noalloc(const uint8_t* d_codes, int64_t row_bytes, int64_t n,
                                    int64_t rows_total, int64_t j0, int64_t j1, const double* d_Y,
                                    int K, int V, const double* d_mean, const double* d_sdinv,
                                    const double* d_left_scale, double* d_accum, double* d_mc,
                                    unsigned* d_status, unsigned long long* d_guards,
                                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LDS_H */
