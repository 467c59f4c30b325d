// Oracle harness: compiles the reference's gwldcore.cpp UNCHANGED (through the
// nanobind-subset shim in oracle/nbshim) and exposes its implementation
// functions through a plain C ABI so tests and the CPU-baseline leg of the
// benchmark can call the reference's own code path.  Test infrastructure only.
//
// Built by oracle/Makefile into oracle/_ref/libref_gwld.so from the sources
// where they lie in the reference tree (src/native/gwldcore.cpp,
// src/native/common/genotype.cpp).
#include "gwldcore.cpp"

#include <cstdio>
#include <string>

namespace {

thread_local std::string g_ref_err;

template <typename T>
nb::object arr(T* p, std::initializer_list<size_t> shape) {
    if (!p) return nb::none();
    return nb::object(nb::ndarray<T>(p, shape));
}

nb::object opt_u64(int has, uint64_t v) {
    return has ? nb::object::from_uint(v) : nb::none();
}

nb::object rows_obj(const int64_t* rows, int64_t n) {
    if (!rows) return nb::none();
    return arr(const_cast<int64_t*>(rows), {(size_t)n});
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_ref_err = e.what();
        return -1;
    }
}

template <typename T>
int phase1_bed(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
               const int64_t* rows, int64_t n_rows, int ddof,
               const T* annot, int64_t L, int64_t K, const T* inv_right,
               int v_start, int v_count, int kmax_hint, const char* rand_dist,
               int has_seed, uint64_t seed, T* Xz, int64_t N, uint8_t* bin_init_mask,
               const char* impute_mode, int has_impute_seed, uint64_t impute_seed,
               T* inv_out) {
    return guarded([&] {
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        phase1_compute_Xz_bed_chunk_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof,
            ann, arr(const_cast<T*>(inv_right), {(size_t)L}), v_start, v_count, kmax_hint,
            rand_dist, opt_u64(has_seed, seed), xz,
            bin_init_mask ? arr(bin_init_mask, {(size_t)K}) : nb::none(), false,
            nb::none(), nb::none(), impute_mode, opt_u64(has_impute_seed, impute_seed),
            nb::none(), inv_out ? arr(inv_out, {(size_t)L}) : nb::none(), 1e-10);
    });
}

template <typename T>
int phase1_geno(T* geno, int64_t N, int64_t L, int blk_start, const T* annot, int64_t K,
                const T* inv_right, int v_start, int v_count, int kmax_hint,
                const char* rand_dist, int has_seed, uint64_t seed, T* Xz,
                uint8_t* bin_init_mask) {
    return guarded([&] {
        nb_mat2f_rw<T> g(geno, {(size_t)N, (size_t)L});
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        phase1_compute_Xz_geno_chunk_impl<T>(
            g, blk_start, ann, arr(const_cast<T*>(inv_right), {(size_t)L}), v_start, v_count,
            kmax_hint, rand_dist, opt_u64(has_seed, seed), xz,
            bin_init_mask ? arr(bin_init_mask, {(size_t)K}) : nb::none(),
            nb::none(), nb::none(), nb::none(), nb::none(), 1e-10);
    });
}

template <typename T>
int phase2_bed(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
               const int64_t* rows, int64_t n_rows, int ddof, const T* inv_left, int64_t L,
               int tile_nvecs, const T* Xz, int64_t N, int64_t Q, T* meansq, int64_t M,
               int N_denom, const char* impute_mode, int has_impute_seed, uint64_t impute_seed,
               double* mc_agg, double* mc_per_snp) {
    return guarded([&] {
        const int64_t K = Q / tile_nvecs;
        nb_mat2f_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        phase2_accum_XtXz_bed_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof,
            nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz, ms,
            nb::none(), nb::none(), N_denom, impute_mode, opt_u64(has_impute_seed, impute_seed),
            mc_agg ? arr(mc_agg, {(size_t)K}) : nb::none(),
            mc_per_snp ? arr(mc_per_snp, {(size_t)M, (size_t)K}) : nb::none());
    });
}

template <typename T>
int phase2_geno(T* geno, int64_t N, int64_t L, int blk_start, const T* inv_left,
                int tile_nvecs, const T* Xz, int64_t Q, T* meansq, int64_t M, int N_denom,
                double* mc_agg, double* mc_per_snp) {
    return guarded([&] {
        const int64_t K = Q / tile_nvecs;
        nb_mat2f_rw<T> g(geno, {(size_t)N, (size_t)L});
        nb_mat2f_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        phase2_accum_XtXz_geno_impl<T>(
            g, blk_start, nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz,
            ms, nb::none(), nb::none(), N_denom,
            mc_agg ? arr(mc_agg, {(size_t)K}) : nb::none(),
            mc_per_snp ? arr(mc_per_snp, {(size_t)M, (size_t)K}) : nb::none());
    });
}

template <typename T>
int resvar_bed(const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
               const int64_t* rows, int64_t n_rows, int ddof, double eps,
               const char* impute_mode, int has_impute_seed, uint64_t impute_seed, T* inv_out) {
    return guarded([&] {
        nb::tuple t = precompute_residual_variances_bed_impl<T>(
            bed_prefix, fam_path, nsnps, step_size, rows_obj(rows, n_rows), ddof, eps, false,
            nb::none(), nb::none(), nb::none(), impute_mode,
            opt_u64(has_impute_seed, impute_seed), nb::none());
        const nb::object o = t[0];
        std::memcpy(inv_out, o.a_.data, sizeof(T) * (size_t)nsnps);
    });
}

template <typename T>
int phase1_bed_rowmajor(const char* bed_prefix, const char* fam_path, int blk_start,
                        int blk_end, const int64_t* rows, int64_t n_rows, int ddof,
                        const T* annot, int64_t L, int64_t K, const T* inv_right, int v_start,
                        int v_count, int kmax_hint, const char* rand_dist, int has_seed,
                        uint64_t seed, T* Xz, int64_t N, const char* impute_mode,
                        int has_impute_seed, uint64_t impute_seed) {
    return guarded([&] {
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2c_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        phase1_compute_Xz_bed_chunk_rowmajor_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof, ann,
            arr(const_cast<T*>(inv_right), {(size_t)L}), v_start, v_count, kmax_hint, rand_dist,
            opt_u64(has_seed, seed), xz, false, nb::none(), nb::none(), impute_mode,
            opt_u64(has_impute_seed, impute_seed), nb::none(), nb::none(), 1e-10);
    });
}

template <typename T>
int col_sums_rowmajor(const T* Xz, int64_t N, int64_t Q, double* out) {
    return guarded([&] {
        nb_mat2c_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        auto r = compute_col_sums_rowmajor_impl<T>(xz);
        std::memcpy(out, r.data(), sizeof(double) * (size_t)Q);
    });
}

template <typename T>
int phase2_mailman_rowmajor(const char* bed_prefix, const char* fam_path, int blk_start,
                            int blk_end, const int64_t* rows, int64_t n_rows, int ddof,
                            const T* inv_left, int64_t L, int tile_nvecs, const T* Xz, int64_t N,
                            int64_t Q, T* meansq, int64_t M, const double* sum_Xz, int N_denom,
                            int has_impute_seed, uint64_t impute_seed, double* mc_agg,
                            double* mc_per_snp) {
    return guarded([&] {
        const int64_t K = Q / tile_nvecs;
        nb_mat2c_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        phase2_accum_XtXz_bed_mailman_rm_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof,
            nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz, ms,
            nb_vec1_ro<double>(const_cast<double*>(sum_Xz), {(size_t)Q}), N_denom,
            opt_u64(has_impute_seed, impute_seed),
            mc_agg ? arr(mc_agg, {(size_t)K}) : nb::none(),
            mc_per_snp ? arr(mc_per_snp, {(size_t)M, (size_t)K}) : nb::none());
    });
}

template <typename T>
int project_rowmajor(T* Xz, int64_t N, int64_t Q, const T* C, const T* R, int64_t p,
                     double* sums) {
    return guarded([&] {
        nb_mat2c_rw<T> xz(Xz, {(size_t)N, (size_t)Q});
        nb::object Co = C ? nb::object(nb::ndarray<const T>(C, {(size_t)N, (size_t)p})) : nb::none();
        nb::object Ro = R ? nb::object(nb::ndarray<const T>(R, {(size_t)p, (size_t)N})) : nb::none();
        auto r = project_rowmajor_inplace_and_col_sums_impl<T>(xz, Co, Ro);
        std::memcpy(sums, r.data(), sizeof(double) * (size_t)Q);
    });
}

template <typename T>
int project_colmajor(T* Xz, int64_t N, int64_t Q, const T* C, const T* R, int64_t p) {
    return guarded([&] {
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)Q});
        nb::object Co = C ? nb::object(nb::ndarray<const T>(C, {(size_t)N, (size_t)p})) : nb::none();
        nb::object Ro = R ? nb::object(nb::ndarray<const T>(R, {(size_t)p, (size_t)N})) : nb::none();
        project_colmajor_inplace_impl<T>(xz, Co, Ro);
    });
}

template <typename T>
int standardize_dosage(T* G, int64_t N, int64_t L, int ddof, double missing, int64_t* nmiss) {
    return guarded([&] {
        nb_mat2f_rw<T> g(G, {(size_t)N, (size_t)L});
        *nmiss = standardize_dosage_inplace_impl<T>(g, ddof, missing, 1);
    });
}

template <typename T>
nb::object matf(const T* p, int64_t r, int64_t c) {
    if (!p) return nb::none();
    return nb::object(nb::ndarray<const T>(p, {(size_t)r, (size_t)c}));
}

// precompute_residual_variances_bed with covariates and snp_var_out.
template <typename T>
int resvar_bed_cov(const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
                   const int64_t* rows, int64_t n_rows, int ddof, double eps,
                   const char* impute_mode, int has_impute_seed, uint64_t impute_seed,
                   const T* C, const T* R, int64_t N, int64_t p, double* snp_var, T* inv_out) {
    return guarded([&] {
        nb::object sv = snp_var ? nb::object(nb::ndarray<double>(snp_var, {(size_t)nsnps})) : nb::none();
        nb::tuple t = precompute_residual_variances_bed_impl<T>(
            bed_prefix, fam_path, nsnps, step_size, rows_obj(rows, n_rows), ddof, eps, false,
            nb::none(), matf(C, N, p), matf(R, p, N), impute_mode,
            opt_u64(has_impute_seed, impute_seed), sv);
        const nb::object o = t[0];
        std::memcpy(inv_out, o.a_.data, sizeof(T) * (size_t)nsnps);
    });
}

// phase1_compute_Xz_bed_chunk with the fused residual variances under covariates.
template <typename T>
int phase1_bed_cov(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
                   const int64_t* rows, int64_t n_rows, int ddof, const T* annot, int64_t L,
                   int64_t K, int v_start, int v_count, const char* rand_dist, uint64_t seed,
                   T* Xz, int64_t N, const char* impute_mode, const T* C, const T* R, int64_t p,
                   const T* gram, T* inv_out) {
    return guarded([&] {
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        nb::object g = gram ? nb::object(nb::ndarray<const T>(gram, {(size_t)p, (size_t)p})) : nb::none();
        phase1_compute_Xz_bed_chunk_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof, ann,
            nb::none(), v_start, v_count, 1, rand_dist, nb::object::from_uint(seed), xz,
            nb::none(), false, matf(C, N, p), matf(R, p, N), impute_mode, nb::none(), g,
            arr(inv_out, {(size_t)L}), 1e-10);
    });
}

}  // namespace

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT const char* ref_last_error() { return g_ref_err.c_str(); }
REF_EXPORT void ref_set_num_threads(int n) {
    set_num_threads(n);
    openblas_set_num_threads(n);
}
REF_EXPORT int ref_get_max_threads() { return get_max_threads(); }
// The reference driver splits threads between OpenMP and BLAS per phase
// (gw_ldscore.py:1765-1771, :2027, :2086): phase 1 runs one BLAS thread per
// OpenMP member, phase 2 one OpenMP thread and a threaded BLAS.
REF_EXPORT void ref_set_omp_threads(int n) { set_num_threads(n); }
REF_EXPORT void ref_set_blas_threads(int n) { openblas_set_num_threads(n); }
REF_EXPORT const char* ref_blas_config() { return openblas_get_config(); }
REF_EXPORT void ref_clear_caches() {
    clear_phase1_csr_cache();
    clear_bed_mapping_cache();
}

#define REF_BOTH(NAME, SIG_F, CALL_F, SIG_D, CALL_D) \
    REF_EXPORT int NAME##_f32 SIG_F { return CALL_F; } \
    REF_EXPORT int NAME##_f64 SIG_D { return CALL_D; }

#define P1_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows, \
    int64_t nr, int ddof, const T* annot, int64_t L, int64_t K, const T* inv, int vs, int vc, \
    int kmax, const char* rd, int hs, uint64_t seed, T* Xz, int64_t N, uint8_t* bim, \
    const char* im, int his, uint64_t iseed, T* inv_out)
#define P1_CALL(T) phase1_bed<T>(bp, fam, bs, be, rows, nr, ddof, annot, L, K, inv, vs, vc, \
    kmax, rd, hs, seed, Xz, N, bim, im, his, iseed, inv_out)
REF_BOTH(ref_phase1_bed, P1_SIG(float), P1_CALL(float), P1_SIG(double), P1_CALL(double))

#define P1G_SIG(T) (T* g, int64_t N, int64_t L, int bs, const T* annot, int64_t K, const T* inv, \
    int vs, int vc, int kmax, const char* rd, int hs, uint64_t seed, T* Xz, uint8_t* bim)
#define P1G_CALL(T) phase1_geno<T>(g, N, L, bs, annot, K, inv, vs, vc, kmax, rd, hs, seed, Xz, bim)
REF_BOTH(ref_phase1_geno, P1G_SIG(float), P1G_CALL(float), P1G_SIG(double), P1G_CALL(double))

#define P2_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows, \
    int64_t nr, int ddof, const T* inv, int64_t L, int tv, const T* Xz, int64_t N, int64_t Q, \
    T* ms, int64_t M, int nd, const char* im, int his, uint64_t iseed, double* mca, double* mcp)
#define P2_CALL(T) phase2_bed<T>(bp, fam, bs, be, rows, nr, ddof, inv, L, tv, Xz, N, Q, ms, M, \
    nd, im, his, iseed, mca, mcp)
REF_BOTH(ref_phase2_bed, P2_SIG(float), P2_CALL(float), P2_SIG(double), P2_CALL(double))

#define P2G_SIG(T) (T* g, int64_t N, int64_t L, int bs, const T* inv, int tv, const T* Xz, \
    int64_t Q, T* ms, int64_t M, int nd, double* mca, double* mcp)
#define P2G_CALL(T) phase2_geno<T>(g, N, L, bs, inv, tv, Xz, Q, ms, M, nd, mca, mcp)
REF_BOTH(ref_phase2_geno, P2G_SIG(float), P2G_CALL(float), P2G_SIG(double), P2G_CALL(double))

#define RV_SIG(T) (const char* bp, const char* fam, int nsnps, int step, const int64_t* rows, \
    int64_t nr, int ddof, double eps, const char* im, int his, uint64_t iseed, T* inv_out)
#define RV_CALL(T) resvar_bed<T>(bp, fam, nsnps, step, rows, nr, ddof, eps, im, his, iseed, inv_out)
REF_BOTH(ref_resvar_bed, RV_SIG(float), RV_CALL(float), RV_SIG(double), RV_CALL(double))

#define P1R_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows, \
    int64_t nr, int ddof, const T* annot, int64_t L, int64_t K, const T* inv, int vs, int vc, \
    int kmax, const char* rd, int hs, uint64_t seed, T* Xz, int64_t N, const char* im, int his, \
    uint64_t iseed)
#define P1R_CALL(T) phase1_bed_rowmajor<T>(bp, fam, bs, be, rows, nr, ddof, annot, L, K, inv, vs, \
    vc, kmax, rd, hs, seed, Xz, N, im, his, iseed)
REF_BOTH(ref_phase1_bed_rowmajor, P1R_SIG(float), P1R_CALL(float), P1R_SIG(double), P1R_CALL(double))

#define CS_SIG(T) (const T* Xz, int64_t N, int64_t Q, double* out)
#define CS_CALL(T) col_sums_rowmajor<T>(Xz, N, Q, out)
REF_BOTH(ref_col_sums_rowmajor, CS_SIG(float), CS_CALL(float), CS_SIG(double), CS_CALL(double))

#define P2M_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows, \
    int64_t nr, int ddof, const T* inv, int64_t L, int tv, const T* Xz, int64_t N, int64_t Q, \
    T* ms, int64_t M, const double* sxz, int nd, int his, uint64_t iseed, double* mca, double* mcp)
#define P2M_CALL(T) phase2_mailman_rowmajor<T>(bp, fam, bs, be, rows, nr, ddof, inv, L, tv, Xz, N, \
    Q, ms, M, sxz, nd, his, iseed, mca, mcp)
REF_BOTH(ref_phase2_mailman_rowmajor, P2M_SIG(float), P2M_CALL(float), P2M_SIG(double), P2M_CALL(double))

#define PRM_SIG(T) (T* X, int64_t N, int64_t Q, const T* C, const T* R, int64_t p, double* sums)
#define PRM_CALL(T) project_rowmajor<T>(X, N, Q, C, R, p, sums)
REF_BOTH(ref_project_rowmajor, PRM_SIG(float), PRM_CALL(float), PRM_SIG(double), PRM_CALL(double))

#define PCM_SIG(T) (T* X, int64_t N, int64_t Q, const T* C, const T* R, int64_t p)
#define PCM_CALL(T) project_colmajor<T>(X, N, Q, C, R, p)
REF_BOTH(ref_project_colmajor, PCM_SIG(float), PCM_CALL(float), PCM_SIG(double), PCM_CALL(double))

#define SDI_SIG(T) (T* G, int64_t N, int64_t L, int ddof, double missing, int64_t* nmiss)
#define SDI_CALL(T) standardize_dosage<T>(G, N, L, ddof, missing, nmiss)
REF_BOTH(ref_standardize_dosage, SDI_SIG(float), SDI_CALL(float), SDI_SIG(double), SDI_CALL(double))

#define RVC_SIG(T) (const char* bp, const char* fam, int nsnps, int step, const int64_t* rows, \
    int64_t nr, int ddof, double eps, const char* im, int his, uint64_t iseed, const T* C, \
    const T* R, int64_t N, int64_t p, double* sv, T* inv_out)
#define RVC_CALL(T) resvar_bed_cov<T>(bp, fam, nsnps, step, rows, nr, ddof, eps, im, his, iseed, \
    C, R, N, p, sv, inv_out)
REF_BOTH(ref_resvar_bed_cov, RVC_SIG(float), RVC_CALL(float), RVC_SIG(double), RVC_CALL(double))

#define P1C_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows, \
    int64_t nr, int ddof, const T* annot, int64_t L, int64_t K, int vs, int vc, const char* rd, \
    uint64_t seed, T* Xz, int64_t N, const char* im, const T* C, const T* R, int64_t p, \
    const T* gram, T* inv_out)
#define P1C_CALL(T) phase1_bed_cov<T>(bp, fam, bs, be, rows, nr, ddof, annot, L, K, vs, vc, rd, \
    seed, Xz, N, im, C, R, p, gram, inv_out)
REF_BOTH(ref_phase1_bed_cov, P1C_SIG(float), P1C_CALL(float), P1C_SIG(double), P1C_CALL(double))

// ---------------------------------------------------------------------------
// Dense-genotype entries with covariates, covariate projections inside the
// BED phases, the legacy direct phase 2, GRM panel products, mu22 and block
// corrections (the reference's own implementations, called unchanged).
// ---------------------------------------------------------------------------
namespace {

template <typename T>
nb::object matf_rw(T* p, int64_t r, int64_t c) {
    if (!p) return nb::none();
    return nb::object(nb::ndarray<T>(p, {(size_t)r, (size_t)c}));
}

template <typename T>
int phase1_geno_cov(T* geno, int64_t N, int64_t L, int blk_start, const T* annot, int64_t K,
                    const T* inv_right, int v_start, int v_count, const char* rand_dist,
                    uint64_t seed, T* Xz, uint8_t* bin_init_mask, const T* C, const T* R,
                    int64_t p, const T* gram, T* inv_out) {
    return guarded([&] {
        nb_mat2f_rw<T> g(geno, {(size_t)N, (size_t)L});
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        nb::object gr = gram ? nb::object(nb::ndarray<const T>(gram, {(size_t)p, (size_t)p})) : nb::none();
        phase1_compute_Xz_geno_chunk_impl<T>(
            g, blk_start, ann, inv_out ? nb::none() : arr(const_cast<T*>(inv_right), {(size_t)L}),
            v_start, v_count, 1, rand_dist, nb::object::from_uint(seed), xz,
            bin_init_mask ? arr(bin_init_mask, {(size_t)K}) : nb::none(), matf(C, N, p),
            matf(R, p, N), gr, inv_out ? arr(inv_out, {(size_t)L}) : nb::none(), 1e-10);
    });
}

template <typename T>
int phase2_geno_cov(T* geno, int64_t N, int64_t L, int blk_start, const T* inv_left,
                    int tile_nvecs, const T* Xz, int64_t Q, T* meansq, int64_t M, const T* C,
                    const T* R, int64_t p, int N_denom, double* mc_agg, double* mc_per_snp) {
    return guarded([&] {
        const int64_t K = Q / tile_nvecs;
        nb_mat2f_rw<T> g(geno, {(size_t)N, (size_t)L});
        nb_mat2f_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        phase2_accum_XtXz_geno_impl<T>(
            g, blk_start, nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz,
            ms, matf(C, N, p), matf(R, p, N), N_denom,
            mc_agg ? arr(mc_agg, {(size_t)K}) : nb::none(),
            mc_per_snp ? arr(mc_per_snp, {(size_t)M, (size_t)K}) : nb::none());
    });
}

template <typename T>
int phase2_bed_cov(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
                   const int64_t* rows, int64_t n_rows, int ddof, const T* inv_left, int64_t L,
                   int tile_nvecs, const T* Xz, int64_t N, int64_t Q, T* meansq, int64_t M,
                   int N_denom, const char* impute_mode, const T* C, const T* R, int64_t p,
                   int mailman, double* mc_agg, double* mc_per_snp) {
    return guarded([&] {
        const int64_t K = Q / tile_nvecs;
        nb_mat2f_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        nb::object ma = mc_agg ? arr(mc_agg, {(size_t)K}) : nb::none();
        nb::object mp = mc_per_snp ? arr(mc_per_snp, {(size_t)M, (size_t)K}) : nb::none();
        if (mailman)
            phase2_accum_XtXz_bed_mailman_impl<T>(
                bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof,
                nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz, ms,
                matf(C, N, p), matf(R, p, N), N_denom, nb::none(), ma, mp);
        else
            phase2_accum_XtXz_bed_impl<T>(
                bed_prefix, fam_path, blk_start, blk_end, rows_obj(rows, n_rows), ddof,
                nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), tile_nvecs, xz, ms,
                matf(C, N, p), matf(R, p, N), N_denom, impute_mode, nb::none(), ma, mp);
    });
}

template <typename T>
int phase1_bed_projright(const char* bed_prefix, const char* fam_path, int blk_start,
                         int blk_end, int ddof, const T* annot, int64_t L, int64_t K,
                         const T* inv_right, int v_start, int v_count, const char* rand_dist,
                         uint64_t seed, T* Xz, int64_t N, uint8_t* bin_init_mask,
                         const char* impute_mode, const T* C, const T* R, int64_t p) {
    return guarded([&] {
        nb_mat2c_ro<T> ann(const_cast<T*>(annot), {(size_t)L, (size_t)K});
        nb_mat2f_rw<T> xz(Xz, {(size_t)N, (size_t)(K * v_count)});
        phase1_compute_Xz_bed_chunk_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, nb::none(), ddof, ann,
            arr(const_cast<T*>(inv_right), {(size_t)L}), v_start, v_count, 1, rand_dist,
            nb::object::from_uint(seed), xz,
            bin_init_mask ? arr(bin_init_mask, {(size_t)K}) : nb::none(), true, matf(C, N, p),
            matf(R, p, N), impute_mode, nb::none(), nb::none(), nb::none(), 1e-10);
    });
}

template <typename T>
int phase2_legacy(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
                  int ddof, const T* inv_left, int64_t L, int nvecs, const T* Xz, int64_t N,
                  int64_t Q, T* meansq, int64_t M, int N_denom, const char* impute_mode,
                  const T* C, const T* R, int64_t p) {
    return guarded([&] {
        const int64_t K = Q / nvecs;
        nb_mat2f_ro<T> xz(const_cast<T*>(Xz), {(size_t)N, (size_t)Q});
        nb_mat2c_rw<T> ms(meansq, {(size_t)M, (size_t)K});
        phase2_compute_XtXz_bed_impl<T>(
            bed_prefix, fam_path, blk_start, blk_end, nb::none(), ddof,
            nb_vec1_ro<T>(const_cast<T*>(inv_left), {(size_t)L}), nvecs, 0, xz, ms,
            matf(C, N, p), matf(R, p, N), N_denom, impute_mode, nb::none());
    });
}

template <typename T>
int apply_grm(const char* bed_prefix, const char* fam_path, int nsnps, int step, int ddof,
              const T* inv_all, const T* panel_in, T* panel_out, int64_t N, int64_t Q,
              const T* C, const T* R, int64_t p, const char* impute_mode, int has_iseed,
              uint64_t iseed, int mailman) {
    return guarded([&] {
        nb_vec1_ro<T> inv(const_cast<T*>(inv_all), {(size_t)nsnps});
        nb_mat2f_ro<T> pin(const_cast<T*>(panel_in), {(size_t)N, (size_t)Q});
        nb_mat2f_rw<T> pout(panel_out, {(size_t)N, (size_t)Q});
        if (mailman)
            apply_grm_bed_panel_mailman_impl<T>(bed_prefix, fam_path, nsnps, step, nb::none(), ddof,
                                                inv, pin, pout, matf(C, N, p), matf(R, p, N),
                                                opt_u64(has_iseed, iseed));
        else
            apply_grm_bed_panel_impl<T>(bed_prefix, fam_path, nsnps, step, nb::none(), ddof, inv,
                                        pin, pout, matf(C, N, p), matf(R, p, N), impute_mode,
                                        opt_u64(has_iseed, iseed));
    });
}

template <typename T>
int resvar_mu22(const char* bed_prefix, const char* fam_path, int nsnps, int step, int ddof,
                const char* impute_mode, const T* annot, int64_t B, const T* C, const T* R,
                int64_t N, int64_t p, T* inv_out, double* mu22) {
    return guarded([&] {
        nb::object ann = nb::object(nb::ndarray<const T>(annot, {(size_t)nsnps, (size_t)B}));
        nb::tuple t = precompute_residual_variances_bed_impl<T>(
            bed_prefix, fam_path, nsnps, step, nb::none(), ddof, 1e-10, true, ann, matf(C, N, p),
            matf(R, p, N), impute_mode, nb::none(), nb::none());
        const nb::object o = t[0];
        std::memcpy(inv_out, o.a_.data, sizeof(T) * (size_t)nsnps);
        const nb::object u = t[1];
        std::memcpy(mu22, u.a_.data, sizeof(double) * (size_t)(B * B));
    });
}

template <typename Tann>
int block_corrections(const double* meansq, int64_t M, int64_t B, const double* mu22,
                      const Tann* annot, int N, double d, double* out4) {
    return guarded([&] {
        nb_mat2c_ro<double> m(const_cast<double*>(meansq), {(size_t)M, (size_t)B});
        nb_mat2c_ro<double> u(const_cast<double*>(mu22), {(size_t)B, (size_t)B});
        nb_mat2c_ro<Tann> a(const_cast<Tann*>(annot), {(size_t)M, (size_t)B});
        nb::tuple t = compute_block_corrections_binary_impl<Tann>(m, u, a, N, d);
        for (int i = 0; i < 4; ++i) {
            const nb::object o = t[i];
            std::memcpy(out4 + (size_t)i * B * B, o.a_.data, sizeof(double) * (size_t)(B * B));
        }
    });
}

}  // namespace

#define P1GC_SIG(T) (T* g, int64_t N, int64_t L, int bs, const T* annot, int64_t K, const T* inv, \
    int vs, int vc, const char* rd, uint64_t seed, T* Xz, uint8_t* bim, const T* C, const T* R,   \
    int64_t p, const T* gram, T* inv_out)
#define P1GC_CALL(T) phase1_geno_cov<T>(g, N, L, bs, annot, K, inv, vs, vc, rd, seed, Xz, bim, C, \
    R, p, gram, inv_out)
REF_BOTH(ref_phase1_geno_cov, P1GC_SIG(float), P1GC_CALL(float), P1GC_SIG(double), P1GC_CALL(double))

#define P2GC_SIG(T) (T* g, int64_t N, int64_t L, int bs, const T* inv, int tv, const T* Xz,      \
    int64_t Q, T* ms, int64_t M, const T* C, const T* R, int64_t p, int nd, double* mca,          \
    double* mcp)
#define P2GC_CALL(T) phase2_geno_cov<T>(g, N, L, bs, inv, tv, Xz, Q, ms, M, C, R, p, nd, mca, mcp)
REF_BOTH(ref_phase2_geno_cov, P2GC_SIG(float), P2GC_CALL(float), P2GC_SIG(double), P2GC_CALL(double))

#define P2BC_SIG(T) (const char* bp, const char* fam, int bs, int be, const int64_t* rows,       \
    int64_t nr, int ddof, const T* inv, int64_t L, int tv, const T* Xz, int64_t N, int64_t Q,     \
    T* ms, int64_t M, int nd, const char* im, const T* C, const T* R, int64_t p, int mailman,     \
    double* mca, double* mcp)
#define P2BC_CALL(T) phase2_bed_cov<T>(bp, fam, bs, be, rows, nr, ddof, inv, L, tv, Xz, N, Q, ms, \
    M, nd, im, C, R, p, mailman, mca, mcp)
REF_BOTH(ref_phase2_bed_cov, P2BC_SIG(float), P2BC_CALL(float), P2BC_SIG(double), P2BC_CALL(double))

#define P1PR_SIG(T) (const char* bp, const char* fam, int bs, int be, int ddof, const T* annot,  \
    int64_t L, int64_t K, const T* inv, int vs, int vc, const char* rd, uint64_t seed, T* Xz,     \
    int64_t N, uint8_t* bim, const char* im, const T* C, const T* R, int64_t p)
#define P1PR_CALL(T) phase1_bed_projright<T>(bp, fam, bs, be, ddof, annot, L, K, inv, vs, vc, rd, \
    seed, Xz, N, bim, im, C, R, p)
REF_BOTH(ref_phase1_bed_projright, P1PR_SIG(float), P1PR_CALL(float), P1PR_SIG(double), P1PR_CALL(double))

#define P2LG_SIG(T) (const char* bp, const char* fam, int bs, int be, int ddof, const T* inv,     \
    int64_t L, int nvecs, const T* Xz, int64_t N, int64_t Q, T* ms, int64_t M, int nd,            \
    const char* im, const T* C, const T* R, int64_t p)
#define P2LG_CALL(T) phase2_legacy<T>(bp, fam, bs, be, ddof, inv, L, nvecs, Xz, N, Q, ms, M, nd,  \
    im, C, R, p)
REF_BOTH(ref_phase2_legacy, P2LG_SIG(float), P2LG_CALL(float), P2LG_SIG(double), P2LG_CALL(double))

#define GRM_SIG(T) (const char* bp, const char* fam, int nsnps, int step, int ddof, const T* inv, \
    const T* pin, T* pout, int64_t N, int64_t Q, const T* C, const T* R, int64_t p,               \
    const char* im, int his, uint64_t iseed, int mailman)
#define GRM_CALL(T) apply_grm<T>(bp, fam, nsnps, step, ddof, inv, pin, pout, N, Q, C, R, p, im,   \
    his, iseed, mailman)
REF_BOTH(ref_apply_grm, GRM_SIG(float), GRM_CALL(float), GRM_SIG(double), GRM_CALL(double))

#define MU22_SIG(T) (const char* bp, const char* fam, int nsnps, int step, int ddof,             \
    const char* im, const T* annot, int64_t B, const T* C, const T* R, int64_t N, int64_t p,      \
    T* inv_out, double* mu22)
#define MU22_CALL(T) resvar_mu22<T>(bp, fam, nsnps, step, ddof, im, annot, B, C, R, N, p,         \
    inv_out, mu22)
REF_BOTH(ref_resvar_mu22, MU22_SIG(float), MU22_CALL(float), MU22_SIG(double), MU22_CALL(double))

#define BCB_SIG(T) (const double* m, int64_t M, int64_t B, const double* u, const T* a, int N,   \
    double d, double* out4)
#define BCB_CALL(T) block_corrections<T>(m, M, B, u, a, N, d, out4)
REF_BOTH(ref_block_corrections, BCB_SIG(float), BCB_CALL(float), BCB_SIG(double), BCB_CALL(double))

// Mailman mean pack statistics (read_block_mailman_mean_memory,
// genotype.cpp:1249-1263): per SNP the observed mean, the pack's inverse
// scale and the observed count, from an in-memory BED image (with header).
REF_EXPORT int ref_mailman_mean_stats(const uint8_t* bed, int64_t bed_size, int n_total,
                                      int64_t bytes_per_snp, int start, int stop,
                                      const int64_t* rows, int64_t n_rows, int ddof,
                                      double* mean, double* inv_std, int* observed) {
    return guarded([&] {
        std::vector<int> r;
        if (rows)
            for (int64_t i = 0; i < n_rows; ++i) r.push_back((int)rows[i]);
        else
            for (int i = 0; i < n_total; ++i) r.push_back(i);
        MailmanPackedBlock pack;
        read_block_mailman_mean_memory(bed, (size_t)bed_size, n_total, (size_t)bytes_per_snp,
                                       start, stop, r, ddof, pack);
        for (int j = 0; j < pack.L; ++j) {
            mean[j] = pack.mean[(size_t)j];
            inv_std[j] = pack.inv_std[(size_t)j];
            observed[j] = pack.observed[(size_t)j];
        }
    });
}
