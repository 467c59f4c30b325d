// Oracle harness: compiles the reference's gxeldcore.cpp UNCHANGED (through the
// nanobind-subset shim in oracle/nbshim) and exposes its MultiEnvironmentKernel
// (source_block, project_sources, target_score_block, normalize_scores), the
// protected right pair and the NumPy-Philox Rademacher generator through a
// plain C ABI, so tests can compare the GPU's GxE products with the
// reference's own code.  Test infrastructure only.
//
// Built by oracle/Makefile into oracle/_ref/libref_gxe.so from the sources
// where they lie in the reference tree (src/native/gxeldcore.cpp,
// src/native/common/genotype.cpp); the build definitions that the reference's
// CMakeLists.txt passes (version strings, GWLDCORE_GEMM_INTEGRITY) are given
// on the command line.
#include "gxeldcore.cpp"

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

template <typename T>
nb_mat2f_ro<T> mat_f(const T* p, int64_t r, int64_t c) {
    return nb_mat2f_ro<T>(p, {(size_t)r, (size_t)c});
}
template <typename T>
nb_vec1_ro<T> vec(const T* p, int64_t n) {
    return nb_vec1_ro<T>(p, {(size_t)n});
}

}  // namespace

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT const char* refg_last_error() { return g_err.c_str(); }

// MultiEnvironmentKernel(environments, feature_basis, feature_power_indices,
// feature_power_offsets, feature_ranks, feature_gram_values,
// feature_gram_offsets, feature_e2_gram_values, common_basis, directions,
// ddof, annotation_bins, threads) (gxeldcore.cpp:10283-10297).
REF_EXPORT int refg_kernel_create(int64_t N, int64_t E, const double* env, int64_t F,
                                  const double* feature_basis, const int64_t* power_idx,
                                  int64_t n_power_idx, const int64_t* power_off,
                                  const int32_t* ranks, const double* gram, int64_t n_gram,
                                  const int64_t* gram_off, const double* e2_gram, int64_t r,
                                  const double* common, const double* directions, int ddof,
                                  int bins, int threads, void** out) {
    return guarded([&] {
        static const double empty = 0.0;
        auto* k = new MultiEnvironmentKernel(
            mat_f(env, N, E), mat_f(feature_basis, N, F), vec(power_idx, n_power_idx),
            vec(power_off, 4 * E + 1), vec(ranks, E), vec(gram, n_gram), vec(gram_off, E + 1),
            vec(e2_gram, n_gram), mat_f(r > 0 ? common : &empty, N, r), mat_f(directions, N, E),
            ddof, bins, threads);
        *out = k;
    });
}

REF_EXPORT void refg_kernel_destroy(void* k) { delete static_cast<MultiEnvironmentKernel*>(k); }

// source_block (gxeldcore.cpp:11008-11240).
REF_EXPORT int refg_source_block(void* k, double* target, int64_t N, int64_t cols,
                                 const double* genotype, int64_t L, const double* probes,
                                 int64_t B, const double* annotation, int64_t K,
                                 const double* scale_x, const double* scale_w, int64_t T,
                                 int env_start, int annotation_is_sqrt) {
    return guarded([&] {
        nb_mat2f_rw<double> tgt(target, {(size_t)N, (size_t)cols});
        static_cast<MultiEnvironmentKernel*>(k)->source_block(
            tgt, mat_f(genotype, N, L), mat_f(probes, L, B), mat_f(annotation, L, K),
            mat_f(scale_x, L, T), mat_f(scale_w, L, T), env_start, annotation_is_sqrt != 0);
    });
}

// project_sources (gxeldcore.cpp:11583-11729); leakages receives one value per
// environment of the tile.
REF_EXPORT int refg_project_sources(void* k, double* panel, int64_t N, int64_t cols,
                                    int columns_per_env, int env_start, double* leakages) {
    return guarded([&] {
        nb_mat2f_rw<double> pn(panel, {(size_t)N, (size_t)cols});
        auto lk = static_cast<MultiEnvironmentKernel*>(k)->project_sources(pn, columns_per_env,
                                                                           env_start);
        std::memcpy(leakages, lk.data(), sizeof(double) * lk.shape(0));
    });
}

// prepare_protected_row_weighted_pair (gxeldcore.cpp:9808): [right, w o right].
REF_EXPORT int refg_prepare_pair(const double* right, int64_t N, int64_t cols,
                                 const double* row_weights, int64_t groups, int threads,
                                 void** out) {
    return guarded([&] {
        auto* p = new ProtectedRightPair(prepare_protected_row_weighted_pair(
            mat_f(right, N, cols), mat_f(row_weights, N, groups), threads));
        *out = p;
    });
}

REF_EXPORT void refg_pair_destroy(void* p) { delete static_cast<ProtectedRightPair*>(p); }

// target_score_block (gxeldcore.cpp:11731-11936); accumulators are
// (E * total_variants) x K row-major and are added to.
REF_EXPORT int refg_target_score_block(void* k, const double* genotype, int64_t N, int64_t L,
                                       void* pair, const double* scale_x, const double* scale_w,
                                       int64_t T, double* axx, double* axw, double* awx,
                                       double* aww, int64_t rows, int64_t K, int block_start,
                                       int total_variants, int probe_count, int env_start) {
    return guarded([&] {
        auto acc = [&](double* p) { return nb_mat2c_rw<double>(p, {(size_t)rows, (size_t)K}); };
        static_cast<MultiEnvironmentKernel*>(k)->target_score_block(
            mat_f(genotype, N, L), *static_cast<ProtectedRightPair*>(pair), mat_f(scale_x, L, T),
            mat_f(scale_w, L, T), acc(axx), acc(axw), acc(awx), acc(aww), block_start,
            total_variants, probe_count, env_start);
    });
}

// normalize_scores (gxeldcore.cpp:12490-12557).
REF_EXPORT int refg_normalize_scores(void* k, double* axx, double* axw, double* awx, double* aww,
                                     int64_t rows, int64_t K, int probe_count) {
    return guarded([&] {
        auto acc = [&](double* p) { return nb_mat2c_rw<double>(p, {(size_t)rows, (size_t)K}); };
        static_cast<MultiEnvironmentKernel*>(k)->normalize_scores(acc(axx), acc(axw), acc(awx),
                                                                  acc(aww), probe_count);
    });
}

// numpy_philox_rademacher_block (gxeldcore.cpp:10070-10113): out is rows x P
// column-major.
REF_EXPORT int refg_philox_rademacher(const uint64_t* keys, int64_t P, int rows, int threads,
                                      double* out) {
    return guarded([&] {
        nb_mat2c_ro<uint64_t> kv(keys, {(size_t)P, 2});
        auto res = numpy_philox_rademacher_block(kv, rows, threads);
        std::memcpy(out, res.data(), sizeof(double) * (size_t)rows * (size_t)P);
    });
}

// ---------------------------------------------------------------------------
// Generalized per-SNP GxE packed products (generalized_gxe_variant.inc:
// 1749-1988).  They are private members of
// GeneralizedGxELDScoreDirectContext, whose constructor needs a whole run's
// tables; the two products read only the context's sample count (rows_) and
// thread count (threads_).  The pointers to those members are obtained
// through explicit template instantiation, which the language lets name
// private members, and the products run on zero-initialized storage with
// just those two fields set.  The reference's code itself is unchanged.
// ---------------------------------------------------------------------------
namespace {

using GenCtx = GeneralizedGxELDScoreDirectContext;

template <typename Tag, typename Tag::type Member>
struct MemberOf {
    friend typename Tag::type member(Tag) { return Member; }
};
struct RowsTag {
    using type = int GenCtx::*;
    friend type member(RowsTag);
};
struct ThreadsTag {
    using type = int GenCtx::*;
    friend type member(ThreadsTag);
};
struct SourceTag {
    using type = void (GenCtx::*)(const MailmanPackedBlock&, const std::vector<double>&, int,
                                  std::vector<double>&) const;
    friend type member(SourceTag);
};
struct TargetTag {
    using type = void (GenCtx::*)(const MailmanPackedBlock&, const double*, int,
                                  std::vector<double>&) const;
    friend type member(TargetTag);
};
template struct MemberOf<RowsTag, &GenCtx::rows_>;
template struct MemberOf<ThreadsTag, &GenCtx::threads_>;
template struct MemberOf<SourceTag, &GenCtx::packed_source_product>;
template struct MemberOf<TargetTag, &GenCtx::packed_target_product>;

}  // namespace

// Mean-imputed Mailman pack of SNPs [start, stop) of an in-memory BED image
// (all n_total samples), then source = packed_source_product(rhs_src) (N x
// cols, column-major; rhs_src L x cols column-major) and target =
// packed_target_product(rhs_tgt) (L x cols; rhs_tgt N x cols), either may be
// skipped with null pointers.
REF_EXPORT int refg_generalized_products(const uint8_t* bed, int64_t bed_size, int n_total,
                                         int64_t bytes_per_snp, int start, int stop, int ddof,
                                         int cols, const double* rhs_src, double* out_src,
                                         const double* rhs_tgt, double* out_tgt) {
    return guarded([&] {
        std::vector<int> rows((size_t)n_total);
        for (int i = 0; i < n_total; ++i) rows[(size_t)i] = i;
        MailmanPackedBlock pack;
        read_block_mailman_mean_memory(bed, (size_t)bed_size, n_total, (size_t)bytes_per_snp,
                                       start, stop, rows, ddof, pack);
        std::vector<unsigned char> storage(sizeof(GenCtx) + alignof(GenCtx), 0);
        void* raw = storage.data();
        size_t space = storage.size();
        auto* ctx = static_cast<GenCtx*>(std::align(alignof(GenCtx), sizeof(GenCtx), raw, space));
        ctx->*member(RowsTag{}) = n_total;
        ctx->*member(ThreadsTag{}) = 1;
        const int L = stop - start;
        std::vector<double> out;
        if (rhs_src && out_src) {
            std::vector<double> rhs(rhs_src, rhs_src + (size_t)L * (size_t)cols);
            (ctx->*member(SourceTag{}))(pack, rhs, cols, out);
            std::memcpy(out_src, out.data(), sizeof(double) * out.size());
        }
        if (rhs_tgt && out_tgt) {
            (ctx->*member(TargetTag{}))(pack, rhs_tgt, cols, out);
            std::memcpy(out_tgt, out.data(), sizeof(double) * out.size());
        }
    });
}
