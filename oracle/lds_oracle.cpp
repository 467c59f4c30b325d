// ORACLE — CPU restatement of the reference's genome-wide LD-score hot path,
// used only as a checker by tests/, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py.  Nothing in the product links or calls it.
//
// Every routine is a plain FP64 restatement of the reference function cited
// beside it (paths relative to the SUMMIT source tree).  Parity of this file
// with the reference itself is pinned by tests/test_oracle_pins.py, which
// runs the reference's own gwldcore.cpp (compiled unchanged by
// oracle/Makefile into oracle/_ref/) on the same inputs.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

// splitmix64 finaliser — genotype.cpp:106-112 (mix64_local).
inline uint64_t mix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// genotype.cpp:114-117 (u01_from_u64).
inline double u01(uint64_t x) {
    return (double)((x >> 11) & ((1ULL << 53) - 1)) * (1.0 / 9007199254740992.0);
}

// HWE imputation — genotype.cpp:133-184.
inline uint64_t hwe_seed_base(uint64_t impute_seed, int global_snp) {
    uint64_t h = mix64(impute_seed);
    h ^= mix64((uint64_t)(uint32_t)global_snp + 0x243f6a8885a308d3ULL);
    return h;
}

inline void hwe_thresholds(long long obs_sum, long long nobs, double& q0, double& q01) {
    double p = 0.0;
    if (nobs > 0) {
        p = (double)obs_sum / (2.0 * (double)nobs);
        if (p < 0.0) p = 0.0;
        if (p > 1.0) p = 1.0;
    }
    q0 = (1.0 - p) * (1.0 - p);
    q01 = q0 + 2.0 * p * (1.0 - p);
}

inline int hwe_value(double q0, double q01, uint64_t seed_base, int global_row) {
    if (q0 >= 1.0) return 0;
    if (q01 <= 0.0) return 2;
    uint64_t h = seed_base;
    h ^= mix64((uint64_t)(uint32_t)global_row + 0x9e3779b97f4a7c15ULL);
    const double u = u01(mix64(h));
    if (u < q0) return 0;
    if (u < q01) return 1;
    return 2;
}

// genotype.cpp:629-649 (compute_mean_invstd_from_completed).
inline void mean_invstd_completed(long long sum, long long sumsq, int n, int ddof,
                                  double& mean, double& inv_std) {
    mean = (n > 0) ? ((double)sum / (double)n) : 0.0;
    inv_std = 1.0;
    const long long denom = (long long)n - (long long)ddof;
    if (n <= 0 || denom <= 0) return;
    double m2 = (double)sumsq - ((double)sum * (double)sum) / (double)n;
    if (m2 < 0.0 && m2 > -1e-12) m2 = 0.0;
    if (m2 > 0.0) {
        const double var = m2 / (double)denom;
        if (var > 0.0 && std::isfinite(var)) inv_std = 1.0 / std::sqrt(var);
    }
}

// genotype.cpp:651-689 (write_mean_imputed_standardized): mean and inverse sd
// over observed calls; missing calls standardize to 0.
inline void mean_invstd_observed(long long nobs, long long sum, long long sumsq, int ddof,
                                 double& mu, double& inv_sd) {
    const double dn = (double)nobs;
    const long long denom = nobs - (long long)ddof;
    mu = (nobs > 0) ? ((double)sum / dn) : 0.0;
    double m2 = 0.0;
    if (nobs > 0) {
        m2 = (double)sumsq - ((double)sum * (double)sum) / dn;
        if (m2 < 0.0 && m2 > -1e-12) m2 = 0.0;
    }
    inv_sd = 1.0;
    if (denom > 0 && m2 > 0.0) {
        const double var = m2 / (double)denom;
        if (var > 0.0) inv_sd = 1.0 / std::sqrt(var);
    }
}

// 2-bit BED code -> value; genotype.cpp:135-140 and :474-574.
inline int code_at(const uint8_t* row, int64_t i) { return (row[i >> 2] >> (2 * (i & 3))) & 3; }

}  // namespace

#define ORC_EXPORT extern "C" __attribute__((visibility("default")))

ORC_EXPORT const char* orc_last_error() { return g_err.c_str(); }

// Standardize SNPs [blk_start, blk_end) of a SNP-major BED image into an
// n_sel x L column-major FP64 block, with the reference's mean or HWE
// imputation.  Restates read_block_standardized_into_impl,
// genotype.cpp:692-952 (decode :474-574, HWE :576-595 and :810-826, mean
// :651-689).  `bed` points at the first SNP row (after the 3-byte header),
// rows are `nbytes` apart; `rows` (sorted, may be null = all) selects samples.
ORC_EXPORT int orc_standardize_block(const uint8_t* bed, int64_t nbytes, int64_t n_total,
                                     const int64_t* rows, int64_t n_sel, int blk_start,
                                     int blk_end, int ddof, int impute_hwe, uint64_t impute_seed,
                                     double* geno, double* mean_out, double* inv_std_out) {
    const int L = blk_end - blk_start;
    const int64_t N = rows ? n_sel : n_total;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < L; ++c) {
        const uint8_t* row = bed + (int64_t)(blk_start + c) * nbytes;
        std::vector<int> code((size_t)N);
        long long nobs = 0, sum = 0, sumsq = 0;
        for (int64_t i = 0; i < N; ++i) {
            const int64_t gi = rows ? rows[i] : i;
            const int b = code_at(row, gi);
            code[(size_t)i] = b;
            if (b != 1) {
                ++nobs;
                if (b == 2) { sum += 1; sumsq += 1; }
                else if (b == 3) { sum += 2; sumsq += 4; }
            }
        }
        double* dst = geno + (int64_t)c * N;
        double mean = 0.0, inv = 1.0;
        if (impute_hwe) {
            long long s = sum, ss = sumsq;
            if (nobs != N) {
                double q0, q01;
                hwe_thresholds(sum, nobs, q0, q01);
                const uint64_t sb = hwe_seed_base(impute_seed, blk_start + c);
                for (int64_t i = 0; i < N; ++i) {
                    if (code[(size_t)i] != 1) continue;
                    const int v = hwe_value(q0, q01, sb, (int)(rows ? rows[i] : i));
                    code[(size_t)i] = (v == 0) ? 0 : (v == 1) ? 2 : 3;
                    s += v;
                    ss += (long long)v * v;
                }
            }
            mean_invstd_completed(s, ss, (int)N, ddof, mean, inv);
            const double g0 = (0.0 - mean) * inv, g1 = (1.0 - mean) * inv, g2 = (2.0 - mean) * inv;
            for (int64_t i = 0; i < N; ++i) {
                const int b = code[(size_t)i];
                dst[i] = (b == 0) ? g0 : (b == 2) ? g1 : g2;
            }
        } else {
            mean_invstd_observed(nobs, sum, sumsq, ddof, mean, inv);
            const double v[4] = {(0.0 - mean) * inv, 0.0, (1.0 - mean) * inv, (2.0 - mean) * inv};
            for (int64_t i = 0; i < N; ++i) dst[i] = v[code[(size_t)i]];
        }
        if (mean_out) mean_out[c] = mean;
        if (inv_std_out) inv_std_out[c] = inv;
    }
    return 0;
}

// Probe block for phase 1: mt19937_64 seeded by make_seed(root, blk_start,
// v_start) (gwldcore.cpp:452-458), drawn column by column
// (gwldcore.cpp:1691-1716).  dist: 0 rademacher (rng()&1 ? +1 : -1),
// 1 gaussian (std::normal_distribution<T>), 2 spherical (gaussian rescaled to
// squared norm L with a long-double sum).  `as_float` selects T = float.
ORC_EXPORT void orc_make_probes(uint64_t root, int blk_start, int v_start, int L, int V,
                                int dist, int as_float, double* Z) {
    uint64_t s = 0x1234abcdULL;
    s ^= mix64(root);
    s ^= mix64((uint64_t)blk_start + 0x9e37ULL);
    s ^= mix64((uint64_t)v_start + 0x85ebULL);
    std::mt19937_64 rng(s);
    std::normal_distribution<float> gf(0.0f, 1.0f);
    std::normal_distribution<double> gd(0.0, 1.0);
    for (int c = 0; c < V; ++c) {
        long double ss = 0.0L;
        double* zc = Z + (int64_t)c * L;
        for (int r = 0; r < L; ++r) {
            double z;
            if (dist == 0) z = (rng() & 1) ? 1.0 : -1.0;
            else z = as_float ? (double)gf(rng) : gd(rng);
            zc[r] = z;
            if (dist == 2) ss += (long double)z * (long double)z;
        }
        if (dist == 2) {
            if (as_float) {
                const float zs = ss > 0.0L ? (float)std::sqrt((long double)L / ss) : 1.0f;
                for (int r = 0; r < L; ++r) zc[r] = (double)((float)zc[r] * zs);
            } else {
                const double zs = ss > 0.0L ? (double)std::sqrt((long double)L / ss) : 1.0;
                for (int r = 0; r < L; ++r) zc[r] *= zs;
            }
        }
    }
}

// Phase 1 for one SNP block: per bin k with members S_k (a_jk > 0, finite,
// inv_j > 0 finite, weight inv_j*sqrt(a_jk) finite; build_phase1_csr
// gwldcore.cpp:1002-1063), Xz[:, k*V+c] = beta*Xz[:, k*V+c]
// + sum_{j in S_k} x_j * z_jc * w_jk, with beta = 0 on a bin's first write
// when bin_init is given (gwldcore.cpp:1768-1838).
ORC_EXPORT int orc_phase1_block(const double* geno, int64_t N, int L, const double* annot,
                                int K, const double* inv, const double* Z, int V, double* Xz,
                                uint8_t* bin_init, int as_float) {
    for (int k = 0; k < K; ++k) {
        std::vector<int> idx;
        std::vector<double> sc;
        for (int i = 0; i < L; ++i) {
            const double a = annot[(int64_t)i * K + k];
            if (a == 0.0 || !(a > 0.0) || !std::isfinite(a)) continue;
            const double iv = inv[i];
            if (!std::isfinite(iv) || iv <= 0.0) continue;
            const double s = iv * std::sqrt(a);
            if (!std::isfinite(s)) continue;
            if (as_float && s > (double)std::numeric_limits<float>::max()) continue;
            idx.push_back(i);
            sc.push_back(s);
        }
        if (idx.empty()) continue;
        double beta = 1.0;
        if (bin_init) {
            beta = bin_init[k] ? 1.0 : 0.0;
            bin_init[k] = 1;
        }
#pragma omp parallel for schedule(static)
        for (int c = 0; c < V; ++c) {
            double* dst = Xz + ((int64_t)k * V + c) * N;
            std::vector<double> acc((size_t)N, 0.0);
            for (size_t r = 0; r < idx.size(); ++r) {
                const double w = Z[(int64_t)c * L + idx[r]] * sc[r];
                const double* x = geno + (int64_t)idx[r] * N;
                for (int64_t n = 0; n < N; ++n) acc[(size_t)n] += x[n] * w;
            }
            // beta = 0 must not read the destination (BLAS semantics: it may
            // hold uninitialized memory, NaN included).
            if (beta == 0.0)
                for (int64_t n = 0; n < N; ++n) dst[n] = acc[(size_t)n];
            else
                for (int64_t n = 0; n < N; ++n) dst[n] += acc[(size_t)n];
        }
    }
    return 0;
}

// Phase 2 for one SNP block: Work = geno^T Xz (L x Q); for each bin segment
// of each Q-panel (32768 columns, gwldcore.cpp:2447-2452, segments
// :2497-2508) upd_j = sum_c Work_jc^2 * inv_j^2 / (N_denom-1)^2, guards
// (non-finite dropped; > 1e10 * segment length dropped; gwldcore.cpp:295-320),
// clamp at 0, meansq[blk_start+j, k] += upd; optional fourth-moment sums
// (gwldcore.cpp:2515-2588).
ORC_EXPORT int orc_phase2_block(const double* geno, int64_t N, int L, int blk_start,
                                const double* inv, int V, const double* Xz, int64_t Q,
                                double* meansq, int K, int N_denom, double* mc_agg,
                                double* mc_per_snp, double extreme_ld_warn, int drop_extreme) {
    if (V <= 0 || Q % V) { g_err = "Xz2d col count must be a multiple of tile_nvecs"; return -1; }
    double denom = (double)N_denom - 1.0;
    if (denom <= 0.0) denom = 1.0;
    const double inv_denom2 = 1.0 / (denom * denom);
    int64_t QP = 32768;
    if (QP > Q) QP = Q;
    QP = (QP / 64) * 64;
    if (QP < 64) QP = (Q < 64) ? Q : 64;
    std::vector<double> work((size_t)L * (size_t)Q);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < L; ++j) {
        const double* x = geno + (int64_t)j * N;
        for (int64_t q = 0; q < Q; ++q) {
            const double* y = Xz + q * N;
            double s = 0.0;
            for (int64_t n = 0; n < N; ++n) s += x[n] * y[n];
            work[(size_t)j * Q + q] = s;
        }
    }
    for (int64_t q0 = 0; q0 < Q; q0 += QP) {
        const int64_t qn = (QP < Q - q0) ? QP : Q - q0;
        int64_t g = q0;
        while (g < q0 + qn) {
            const int64_t k = g / V;
            const int64_t vin = g - k * V;
            const int64_t len = std::min<int64_t>(q0 + qn - g, V - vin);
            double agg = 0.0;
            for (int j = 0; j < L; ++j) {
                double acc = 0.0, acc2 = 0.0;
                for (int64_t c = 0; c < len; ++c) {
                    const double w = work[(size_t)j * Q + g + c];
                    acc += w * w;
                    acc2 += (w * w) * (w * w);
                }
                const double iv = inv[j];
                const double sc = (std::isfinite(iv) && iv > 0.0) ? iv * iv * inv_denom2 : 0.0;
                double upd = acc * sc;
                const bool nonfinite = !std::isfinite(upd);
                const bool extreme = !nonfinite && std::isfinite(extreme_ld_warn) &&
                                     upd > extreme_ld_warn * (double)len;
                if (nonfinite || (extreme && drop_extreme)) continue;
                if (upd < 0.0) upd = 0.0;
                meansq[(int64_t)(blk_start + j) * K + k] += upd;
                const double s2 = acc2 * sc * sc;
                agg += s2;
                if (mc_per_snp) mc_per_snp[(int64_t)(blk_start + j) * K + k] += s2;
            }
            if (mc_agg) mc_agg[k] += agg;
            g += len;
        }
    }
    return 0;
}

// Inverse residual sd without covariates: inv_j = 1/sqrt(max(eps,
// ||x_j||^2/(N-1))) (compute_inv_resvar_from_geno_block, gwldcore.cpp:3220-3333).
ORC_EXPORT void orc_inv_resvar_block(const double* geno, int64_t N, int L, double eps,
                                     double* inv_out) {
    for (int j = 0; j < L; ++j) {
        const double* x = geno + (int64_t)j * N;
        double acc = 0.0;
        for (int64_t n = 0; n < N; ++n) acc += x[n] * x[n];
        const double var = acc / (double)(N - 1);
        const double safe = std::isnan(var) ? var : (var > eps ? var : eps);
        inv_out[j] = 1.0 / std::sqrt(safe);
    }
}

// Integer product checker for the GPU kernels' exact parts: out[j*Q+q] =
// sum_i g_ij * y[q*N+i] with g decoded from the BED image (missing -> 0) and
// `obs[j*Q+q]` = sum over observed samples of y.  Exact in int64.
ORC_EXPORT void orc_int_products(const uint8_t* bed, int64_t nbytes, int64_t N, int L,
                                 const int8_t* y, int64_t Q, int64_t* out, int64_t* obs) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < L; ++j) {
        const uint8_t* row = bed + (int64_t)j * nbytes;
        for (int64_t q = 0; q < Q; ++q) {
            int64_t s = 0, so = 0;
            for (int64_t i = 0; i < N; ++i) {
                const int b = code_at(row, i);
                const int64_t v = y[q * N + i];
                if (b != 1) so += v;
                s += (b == 2 ? 1 : b == 3 ? 2 : 0) * v;
            }
            out[(int64_t)j * Q + q] = s;
            if (obs) obs[(int64_t)j * Q + q] = so;
        }
    }
}

// The seeded synthetic genotype generator of summit_b200/bedfile.py, in C for
// CPU-side sample generation (identical bytes): packed rows of ceil(n/4).
ORC_EXPORT void orc_synth_bed(int64_t n, int64_t M, uint64_t seed, const int64_t* t0,
                              const int64_t* t1, int missing, uint8_t* out) {
    const uint64_t k2 = mix64(seed ^ mix64(2ULL));
    const uint64_t k3 = mix64(seed ^ mix64(3ULL));
    const int64_t nb = (n + 3) / 4;
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; ++b) {
        long long u[4] = {0, 0, 0, 0};
        for (int64_t j = 0; j < M; ++j) {
            uint32_t byte = 0;
            for (int t = 0; t < 4; ++t) {
                const int64_t i = b * 4 + t;
                if (i >= n) break;
                const uint64_t r = mix64(k2 ^ mix64(((uint64_t)j << 32) | (uint64_t)i));
                const long long e = (long long)(r & 0xFFFFULL) + (long long)((r >> 16) & 0xFFFFULL) +
                                    (long long)((r >> 32) & 0xFFFFULL) + (long long)(r >> 48) -
                                    131070LL;
                u[t] = (j == 0) ? e : ((58982LL * u[t] + 28567LL * e) >> 16);
                uint32_t code = (u[t] < t0[j]) ? 0u : (u[t] < t1[j]) ? 2u : 3u;
                if (missing &&
                    (mix64(k3 ^ mix64(((uint64_t)j << 32) | (uint64_t)i)) >> 32) < 42949673ULL)
                    code = 1u;
                byte |= code << (2 * t);
            }
            out[j * nb + b] = (uint8_t)byte;
        }
    }
}

ORC_EXPORT int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
