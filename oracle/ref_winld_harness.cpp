// Oracle harness: compiles the reference's winldcore.cpp UNCHANGED (through the
// nanobind-subset shim in oracle/nbshim) and exposes compute_windowed_ld_chr
// and compute_maf_bed through a plain C ABI, so tests can compare the GPU's
// exact windowed LD scores with the reference's own code.  Test infrastructure
// only.
//
// Built by oracle/Makefile into oracle/_ref/libref_winld.so from the sources
// where they lie in the reference tree (src/native/winldcore.cpp,
// src/native/common/genotype.cpp).
#include "winldcore.cpp"

#include <cstring>
#include <string>

namespace {

thread_local std::string g_err;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

nb::object rows_obj(const int64_t* rows, int64_t n) {
    if (!rows) return nb::none();
    return nb::object(nb::ndarray<int64_t>(const_cast<int64_t*>(rows), {(size_t)n}));
}

}  // namespace

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT const char* refw_last_error() { return g_err.c_str(); }
REF_EXPORT void refw_set_num_threads(int n) {
    set_num_threads(n);
    openblas_set_num_threads(n);
}

// compute_windowed_ld_chr (winldcore.cpp:972-987).  annot is m x K
// column-major; out (m x K column-major) receives the returned array.
// C (N x p, column-major) and R (p x N, column-major) may be NULL.
REF_EXPORT int refw_compute_windowed_ld_chr(const char* bed_prefix, const char* fam_path,
                                            int chr_start, int chr_end, const int64_t* bp,
                                            const double* annot, int64_t K, double ld_wind_kb,
                                            int chunk_size, const int64_t* rows, int64_t n_rows,
                                            const double* C, const double* R, int64_t N, int64_t p,
                                            const char* impute_mode, int has_impute_seed,
                                            uint64_t impute_seed, int panel_cols, int cache_mb,
                                            double* out) {
    return guarded([&] {
        const size_t m = (size_t)(chr_end - chr_start);
        nb_vec1_ro<int64_t> bpv(bp, {m});
        nb_mat2f_ro<double> ann(annot, {m, (size_t)K});
        nb::object Co = nb::none(), Ro = nb::none();
        if (C && R) {
            Co = nb::object(nb::ndarray<const double>(C, {(size_t)N, (size_t)p}));
            Ro = nb::object(nb::ndarray<const double>(R, {(size_t)p, (size_t)N}));
        }
        nb::object seed = has_impute_seed ? nb::object::from_uint(impute_seed) : nb::none();
        auto res = compute_windowed_ld_chr_impl(bed_prefix, fam_path, chr_start, chr_end, bpv, ann,
                                                ld_wind_kb, chunk_size, rows_obj(rows, n_rows), Co,
                                                Ro, impute_mode, seed, panel_cols, cache_mb);
        std::memcpy(out, res.data(), sizeof(double) * m * (size_t)K);
    });
}

// compute_maf_bed (winldcore.cpp:988-993).
REF_EXPORT int refw_compute_maf_bed(const char* bed_prefix, const char* fam_path, int nsnps,
                                    int step_size, const int64_t* rows, int64_t n_rows,
                                    double* out) {
    return guarded([&] {
        auto res = compute_maf_bed_impl(bed_prefix, fam_path, nsnps, step_size,
                                        rows_obj(rows, n_rows));
        std::memcpy(out, res.data(), sizeof(double) * (size_t)nsnps);
    });
}
