// Internal interfaces between the host orchestration (lds_host.cu) and the
// kernels (lds_kernels.cu).  Not part of the C ABI.
#pragma once
#include <atomic>
#include <cstdint>
#include <string>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

namespace lds {

// Padding rules of the device genotype image.
constexpr int kSamplePad = 256;   // N_pad multiple (phase-2 K-steps, phase-1 sample tiles)
constexpr int kSnpPad = 128;      // M_pad multiple (phase-2 SNP tiles)
constexpr int kColTile = 16;      // probe columns per tile (bins padded to a multiple)
constexpr int kSnpStep = 32;      // phase-1 K-step (SNPs); CSR lists padded to a multiple
constexpr int kMaxSlices = 6;

// Device-resident, padded genotype image: SNP-major 2-bit codes, row stride
// nbp = N_pad/4 bytes, M_pad rows.  Padding samples and rows hold code 01
// (missing), so they decode to g = 0, o = 0 and contribute nothing.
struct DevGeno {
    int64_t N = 0, N_pad = 0, nbp = 0, M = 0, M_pad = 0;
    uint8_t* codes = nullptr;
};

// Per-SNP code counts produced by the stats kernel: n0, n1, n2, nmiss
// (real samples only).
struct SnpCounts {
    int32_t n[4];
};

// ---- kernel launchers (all on `st`) ----
// Repack raw BED rows (row stride src_bytes, n_total samples) into the padded
// device layout, selecting `rows` (device int32, may be null = all).
void launch_repack(const uint8_t* src, int64_t src_bytes, int64_t n_total, const int32_t* rows,
                   const DevGeno& g, cudaStream_t st);
void launch_counts(const DevGeno& g, SnpCounts* out, cudaStream_t st);
// HWE imputation in place (genotype.cpp:146-184, :810-826): q0/q01/seed_base
// per SNP (host-computed doubles), global row index per selected sample.
void launch_hwe_impute(const DevGeno& g, const double* q0, const double* q01,
                       const uint64_t* seed_base, const int32_t* global_rows, cudaStream_t st);

// Phase-1 weights: for each bin k and probe v, W1[r] = s_j * sc_r * z_{j v}
// and W2[r] = mu_j * W1[r] over the bin's CSR members (j = rowind[r]);
// quantized per column into S signed int8 digits with a power-of-two scale.
struct P1Weights {
    int K = 0, V = 0, Vp = 0, S = 4;
    const int32_t* rowind = nullptr;     // concatenated member lists (padded per bin)
    const double* sc = nullptr;          // inv_j * sqrt(a_jk) per member (0 in padding)
    const int64_t* bin_off = nullptr;    // K+1 offsets into rowind/sc (multiples of kSnpStep)
    const int64_t* wq_off = nullptr;     // K offsets (bytes) into wq
    int8_t* wq = nullptr;                // per bin: [S][2][Vp][nnzp]
    double* colscale = nullptr;          // K*Vp
};
void launch_p1_weights(const P1Weights& w, const double* mean, const double* sdinv,
                       const double* Z, int64_t z_ld, int64_t z_row0, cudaStream_t st);

// Phase 1: Y[:, k*V+v] = sum_r x_{rowind[r]} * W[r, (k,v)], FP64 output
// (N_pad rows, column stride N_pad, only real columns written).
void launch_p1(const DevGeno& g, const P1Weights& w, const int64_t* h_bin_off, double* Y,
               cudaStream_t st);

// Quantize Y (N_pad x K*V, FP64) into S int8 digit planes Yq[S][K*Vp][N_pad]
// with per-column power-of-two scales (padding columns -> 0).
void launch_quantize_y(const double* Y, int64_t N, int64_t N_pad, int K, int V, int Vp, int S,
                       int8_t* Yq, double* colscale, cudaStream_t st);

// Phase 2 over SNP rows [j0, j1): Work = x_j^T Y, per bin k:
// upd = sum_v Work^2 * left_scale_j with guards; accum[(j-j0_out)*K + k] += upd;
// mc (may be null) += sum_v Work^4 * left_scale^2.  guard_counts[0..1] +=
// dropped non-finite / extreme counts.
struct P2Args {
    int K = 0, V = 0, Vp = 0, S = 4;
    int64_t j0 = 0, j1 = 0, out_row0 = 0;
    const int8_t* Yq = nullptr;
    const double* colscale = nullptr;
    const double* mean = nullptr;
    const double* sdinv = nullptr;
    const double* left_scale = nullptr;
    double* accum = nullptr;
    double* mc = nullptr;
    unsigned long long* guard_counts = nullptr;
    double extreme_warn = 1e10;
    int drop_extreme = 1;
    // Verification mode (S must be 1): write exact int64 G^T y / O^T y of the
    // single bin to raw_g / raw_o ((j - out_row0) * V + v) instead of reducing.
    long long* raw_g = nullptr;
    long long* raw_o = nullptr;
};
void launch_p2(const DevGeno& g, const P2Args& a, cudaStream_t st);

// Synthetic generator (bedfile.py), writing n samples x M SNPs, row stride
// ceil(n/4), into `out` (device).
void launch_synth(int64_t n, int64_t M, uint64_t seed, const int64_t* t0, const int64_t* t1,
                  int missing, uint8_t* out, cudaStream_t st, int64_t ld = 0, int pad_missing = 0);

// Exact products with the D nearest right-hand neighbours (lds_band.cu):
// counts[(j (D+1) + d) 4 + {0..3}] = GG, GO, OG, OO integer sums of SNPs j, j+d;
// xx[j (D+1) + d] = x_j . x_{j+d} in FP64 from them.
void launch_nn_band(const DevGeno& g, int D, int32_t* counts, cudaStream_t st);
void launch_nn_band_finish(int64_t M, int D, const int32_t* counts, const double* mean,
                           const double* sdinv, double* xx, cudaStream_t st);

// Exact windowed LD scores (lds_gram.cu).  Work item x: tile J = SNPs
// [x.x, x.x + 128), partner tiles I = [x.y + 128 t, +128) for t < x.z, sums
// into partial slot x.w.  lo/hi: partner interval of SNP j at (j - row0);
// mean/rs (1/sqrt(c_jj), 0 for a constant SNP) indexed by SNP; annot row-major
// ((i - row0) K + b); corr_den = 1/(corr_dim - 1) for the unbiased r^2, 0 for r^2.
struct GramArgs {
    int nkt = 0, K = 0;
    int64_t row0 = 0, row1 = 0;
    const int4* items = nullptr;
    const int32_t* lo = nullptr;
    const int32_t* hi = nullptr;
    const double* mean = nullptr;
    const double* rs = nullptr;
    const double* annot = nullptr;
    double corr_den = 0.0;
    double* partial = nullptr;      // (slot 128 + jl) K + b, zeroed by the caller
    unsigned* status = nullptr;
};
size_t gram_ld_smem_bytes();
void launch_gram_ld(const CUtensorMap& tmC, const GramArgs& a, int n_items, cudaStream_t st);
// out[(j - row0) ld_row + b ld_col] = sum of tile (j - row0)/128's slots
// [slot_beg[T], slot_beg[T+1]) in order.
void launch_gram_reduce(const double* partial, const int32_t* slot_beg, int64_t row0, int64_t row1,
                        int K, double* out, int64_t ld_row, int64_t ld_col, cudaStream_t st);

// GxE (lds_gxe.cu): see the file header for the column layouts.
void launch_gxe_source_finalize(const double* Y, int64_t N, int64_t N_pad, int64_t C, int cols_half,
                                const double* env, int64_t env_ld, int env_start, double* target,
                                int64_t t_ld, cudaStream_t st);
// out[c nb + a] = basis_a . panel_c (basis null: column sums, nb = 1); with
// `squares` out[c] = panel_c . panel_c.  nb <= col_dots_max_basis().
void launch_col_dots(const double* panel, int64_t p_ld, int64_t N, int64_t C, const double* basis,
                     int64_t b_ld, int nb, int squares, double* out, cudaStream_t st);
int col_dots_max_basis();
// panel_c -= sum_a basis_a coef[c nb + a] (the last basis column is all ones,
// scaled by last_scale, when ones_last).
void launch_sub_lowrank(double* panel, int64_t ld, int64_t N, int64_t C, const double* basis,
                        int64_t b_ld, int nb, const double* coef, int ones_last, double last_scale,
                        cudaStream_t st);
void launch_gxe_pair(const double* S, int64_t s_ld, int64_t N, int64_t N_pad, int64_t C,
                     int64_t cols_per_group, const double* w, int64_t w_ld, int w_first,
                     double* Ypair, cudaStream_t st);
void launch_gxe_target_finalize(const double* S, int64_t L, int Kp, int K, int T, const double* sx,
                                const double* sw, int64_t s_ld, const int32_t* ranks, int64_t N,
                                int env_start, int64_t total, int64_t block_start, double* a0,
                                double* a1, double* a2, double* a3, cudaStream_t st);
void launch_scale(double* x, int64_t n, double s, cudaStream_t st);
void launch_gxe_check(const double* probes, int64_t np, const double* sx, const double* sw,
                      int64_t ns, const double* annot, int64_t na, unsigned* flag, cudaStream_t st);
void launch_philox_rademacher(const uint64_t* keys, int64_t P, int64_t rows, double* out,
                              cudaStream_t st);

// Sketch-panel utilities (lds_proj.cu), T = float or double.
template <typename T> void launch_col_sums_rowmajor(const T* X, int64_t N, int64_t Q, double* out,
                                                    cudaStream_t st);
template <typename T> void launch_rowmajor_to_colmajor(const T* in, int64_t N, int64_t Q,
                                                       double* out, cudaStream_t st);
template <typename T> void launch_colmajor_to_rowmajor(const double* in, int64_t N, int64_t Q,
                                                       T* out, cudaStream_t st);
template <typename T> void launch_convert(const T* in, int64_t n, double* out, cudaStream_t st);
template <typename T> void launch_convert_back(const double* in, int64_t n, T* out,
                                               cudaStream_t st);
template <typename T> void launch_standardize_dosage(T* G, int64_t N, int64_t L, int ddof,
                                                     double missing, unsigned long long* counts,
                                                     cudaStream_t st);

// Generalized per-variant GxE estimator (lds_generalized.cu): the global
// variant x probe sign stream (out column-major L x B; root_state = splitmix64
// of root ^ namespace key ^ the root constant) and the component-kernel
// diagonals for at most kGenMaxQ context bases and kGenMaxR fixed effects.
constexpr int kGenMaxQ = 6;
constexpr int kGenMaxR = 16;
void launch_global_probes(uint64_t root_state, int64_t v0, int64_t L, int64_t p0, int64_t B,
                          double* out, cudaStream_t st);
// Pass-2 scores of a variant block (one CTA per row; the row's K*B*F cross
// sketches in shared memory, at most kGenRowsMaxSmem bytes) and the directed
// numerator accumulation.
constexpr int kGenRowsMaxSmem = 200 * 1024;
size_t gen_rows_smem_bytes(int cols);
void launch_gen_project(const double* base, const double* basis, int Q, const double* fixed,
                        int R, int K, int B, int64_t N, double* out, double* leak, double* pn2,
                        cudaStream_t st);
void launch_gen_assemble_rhs(const double* S, int64_t Np, const double* basis, int Q,
                             const int* fam_t, const int* fam_s, int K, int B, int F, int64_t N,
                             double* Y, cudaStream_t st);
void launch_gen_rows(const long long* raw_g, const long long* raw_o, int64_t raw_ld,
                     const double* cs, const double* mean, const double* sdinv, int64_t j0,
                     int64_t L, double inv_rr, int K, int B, int F, int P, const int* term_off,
                     const int* term_f1, const int* term_f2, double* out, cudaStream_t st);
void launch_gen_directed(const double* rows, int64_t L, const double* annot, int64_t j0, int K,
                         int P, double* directed, cudaStream_t st);
void launch_component_diag(const uint8_t* codes, int64_t nbp, const double* mean,
                           const double* sdinv, int64_t j0, int64_t L, int64_t N,
                           const double* annot, int K, const double* basis, int Q,
                           const double* fixed, int R, const double* coef, const int* pq,
                           const int* pr, const double* kf, int P, double* num, cudaStream_t st);

// Phase-2 product checksums (lds_check.cu): u[wl][i] over the n_windows
// windows of a batch (K super-bins each, V probes from global probe v0), and
// rhs[2j], rhs[2j+1] += sum_i g_ij u(i), sum_i o_ij u(i) for the rows of each tile.
void launch_check_u(const int8_t* yq, int64_t yq_cols, int ncolp, int K, int V, int v0,
                    int64_t n_windows, int64_t N_pad, unsigned long long* u, cudaStream_t st);
void launch_check_rhs(const uint8_t* codes, int64_t nbp, const int4* tiles, int64_t n_tiles, int K,
                      const unsigned long long* u, int64_t N_pad, unsigned long long* rhs,
                      cudaStream_t st);

// Jackknife and normal-equation solves (lds_jack.cu).
int sym_solve_max_k();
void launch_block_sums(const double* X, int64_t P, const int64_t* starts, const int64_t* ends,
                       int64_t B, double* out, cudaStream_t st);
void launch_delete_one(const double* blocks, int64_t B, int64_t P, double* sys, cudaStream_t st);
// Optional per-system outputs of the symmetric solve (device pointers, each
// may be null): eigenvectors (K x K, column p for the p-th smallest
// eigenvalue), residual S x - b (K), symmetry error and tolerance (1 each).
struct SymSolveExtras {
    double* evec = nullptr;
    double* resid = nullptr;
    double* asym = nullptr;
    double* tol = nullptr;
};
void launch_sym_solve(const double* sys, int64_t nsys, int K, double rtol, int require_full_rank,
                      double* x, int* rank, double* eig, int* status, cudaStream_t st,
                      const SymSolveExtras& ex = SymSolveExtras());
void launch_jackknife_stats(const double* reps, int64_t R, int K, double* mean, double* se,
                            double* cov, cudaStream_t st);

// Near-field control variate sums (lds_cv.cu): C[j K + k] += sum_v a_jkv^2 and,
// if mu is set, mu[j K + k] = E[a_jk^2]; D in {4, 8, 15}.
struct CvNearArgs {
    int64_t M = 0;
    int K = 0, V = 0;
    const double* z = nullptr;      // probes, z[v z_ld + i]
    int64_t z_ld = 0;
    const double* annot = nullptr;  // M x K row-major
    const int32_t* win_of = nullptr;
    const double* sqrt_ls = nullptr;
    const double* xx = nullptr;     // M x (D+1) neighbour products
    double* C = nullptr;
    double* mu = nullptr;
    double* C2 = nullptr;           // if set, probes v >= split_v add to C2 instead of C
    int split_v = 0;
};
void launch_cv_near(const CvNearArgs& a, int D, cudaStream_t st);
// Windowed finalize: meansq = sum of `slices` slices of acc (each M*K), and
// ld = meansq / nvecs - mkw[win_of[j] K + k] / nd.
void launch_win_finalize(const double* acc, int slices, int64_t M, int K, double nvecs, double nd,
                         const int32_t* win_of, const double* mkw, double* ld, double* meansq,
                         cudaStream_t st);

// Surrogate network of the learned control variate (lds_mlp.cu): in -> 128 ->
// 128 -> 128 -> out, GELU, FP32 master parameters laid out as below.
constexpr int kMlpHidden = 128;
struct MlpLayout {
    int64_t W1, b1, W2, b2, W3, b3, W4, b4, total;
};
__host__ __device__ inline MlpLayout mlp_layout(int in, int out) {
    MlpLayout L;
    L.W1 = 0;
    L.b1 = L.W1 + (int64_t)kMlpHidden * in;
    L.W2 = L.b1 + kMlpHidden;
    L.b2 = L.W2 + (int64_t)kMlpHidden * kMlpHidden;
    L.W3 = L.b2 + kMlpHidden;
    L.b3 = L.W3 + (int64_t)kMlpHidden * kMlpHidden;
    L.W4 = L.b3 + kMlpHidden;
    L.b4 = L.W4 + (int64_t)out * kMlpHidden;
    L.total = L.b4 + out;
    return L;
}
__host__ __device__ inline int mlp_out_pad(int out) { return (out + 3) & ~3; }
struct MlpArgs {
    const float* params = nullptr;
    int in = 0, out = 0;
};
// BF16 weight copies for the products (mlp_pack_elems bf16 values), remade
// whenever the parameters change.
size_t mlp_pack_elems(int in, int out);
void launch_mlp_pack(const MlpArgs& a, void* pack, cudaStream_t st);
// Forward over n rows (x rows gathered through `rows` if set): out (n x out,
// may be null); with `target`, dout (n x out_pad) = 2 (o - t) gscale and
// loss += gscale sum (o - t)^2; zs (n x 3 x 128, may be null) keeps z1..z3.
void launch_mlp_forward(const MlpArgs& a, const void* pack, const float* x, const int32_t* rows,
                        int64_t n, const float* target, float* out, float* zs, float* dout,
                        double* loss, float gscale, cudaStream_t st);
// Backward: grad (zeroed by the caller) += d loss / d params.
void launch_mlp_backward(const MlpArgs& a, const void* pack, const float* x, const int32_t* rows,
                         int64_t n, const float* zs, const float* dout, float* dzs, float* grad,
                         cudaStream_t st);
void launch_mlp_adam(float* p, float* m, float* v, const float* g, int64_t P, float lr, float b1,
                     float b2, float eps, float bc1, float bc2, cudaStream_t st);

// Launch accounting.
// ---- device Rademacher probe streams (lds_probes.cu) ----
// One std::mt19937_64 stream per unit: its L x V block (column-major, rows
// row0 .. row0 + L of Z with leading dimension ld) in stream order.
struct ProbeUnit {
    int64_t row0;
    int32_t L;
    int32_t pad;
    uint64_t seed;
};
void launch_rademacher_units(const ProbeUnit* units, int64_t n_units, int V, double* Z, int64_t ld,
                             cudaStream_t st);

// ---- dense FP64 work (lds_dense.cu) ----
// C[m, n] = alpha sum_k A(m, k) B(k, n) + beta C[m, n] with
// A(m, k) = A[m a_ms + kk a_ks] (kk = a_kidx[k] when a_kidx is set; squared
// when a_square), B(k, n) = B[k b_ks + n b_ns], C[m c_ms + n c_ns]; beta == 0
// does not read C.
struct DGemmArgs {
    int64_t M = 0, N = 0, K = 0;
    const double* A = nullptr;
    int64_t a_ms = 1, a_ks = 1;
    const int32_t* a_kidx = nullptr;
    int a_square = 0;
    const double* B = nullptr;
    int64_t b_ks = 1, b_ns = 1;
    double* C = nullptr;
    int64_t c_ms = 1, c_ns = 1;
    double alpha = 1.0, beta = 0.0;
};
void launch_dgemm(const DGemmArgs& a, cudaStream_t st);
void launch_dense_p2_epilogue(const double* W, int64_t L, int K, int V, const double* ls,
                              double* accum, double* mc, unsigned long long* guards,
                              double extreme_warn, int drop_extreme, cudaStream_t st);
void launch_decode_standardized(const DevGeno& g, int64_t j0, int64_t L, const double* mean,
                                const double* sdinv, double* X, int64_t ldx, cudaStream_t st);
void launch_col_sumsq(const double* X, int64_t N, int64_t ld, int64_t L, double* ss,
                      cudaStream_t st);
void launch_restandardize_cols(double* X, int64_t N, int64_t ld, int64_t L, cudaStream_t st);
int window_cov_max_bins();
void launch_window_cov_epilogue(const double* S, int64_t rows, int64_t p0, const int64_t* lo,
                                const int64_t* hi, const double* annot, int64_t annot_row0, int K,
                                double invN, double corr_den, double* out, cudaStream_t st);
template <typename Tann>
void launch_block_corrections(const double* meansq, const double* mu22, const Tann* annot,
                              int64_t M, int B, double N, double d, double* R2, double* rho2,
                              double* bias, double* delta, cudaStream_t st);

void count_launch();

// Set the text returned by lds_last_error() for the calling thread.
void set_last_error(const std::string& msg);

// Phase-2 guard settings from the environment, read once per process like
// the reference's (gwldcore.cpp:295-308): SUMMIT_P2_EXTREME_LD_WARN (or
// SUMMIT_P2_ABS_LD_MAX; default 1e10, <= 0 disables) and
// SUMMIT_P2_DROP_EXTREME (default on).
double phase2_extreme_warn();
int phase2_drop_extreme();

// Setters of the per-file copies of the bounded-wait iteration limit of the
// tensor-core kernels (lds_tc.cuh); each applies to the current device.
using WaitLimitSetter = cudaError_t (*)(long long);
void register_wait_limit_setter(WaitLimitSetter f);
// Calls every registered setter; returns the first error.
cudaError_t set_wait_limit_all(long long iters);
// Bounds-checked builds (-DLDS_CHECKED): setters of the per-file device
// pointers to the error word that failed index checks write (lds_tc.cuh).
using CheckedErrSetter = cudaError_t (*)(unsigned*);
void register_checked_err_setter(CheckedErrSetter f);
std::vector<CheckedErrSetter>& checked_err_setters();
// Self-test of the bounded wait (lds_umma.cu): one thread waits on an
// mbarrier that nothing arrives at; *status_dev = 1 when the wait ran out,
// 2 if it (wrongly) completed.
void launch_wait_timeout_probe(unsigned* status_dev, cudaStream_t st);

// Run `set` (a cudaFuncSetAttribute call) once for each device it is needed
// on.  Function attributes apply to the current device only, so a process
// that drives several GPUs must set them on every one; `done` holds one bit
// per device id.  Two threads racing here may both call `set`, which is
// harmless (the attribute call is idempotent).
template <typename F>
inline void once_per_device(std::atomic<unsigned long long>& done, F&& set) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set();
        return;
    }
    const unsigned long long bit = 1ULL << dev;
    if (done.load(std::memory_order_acquire) & bit) return;
    set();
    done.fetch_or(bit, std::memory_order_acq_rel);
}

}  // namespace lds
