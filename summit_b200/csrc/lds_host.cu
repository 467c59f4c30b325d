// Host side of liblds.so: C ABI (include/lds.h), device genotype cache,
// per-SNP statistics, probe streams, and the phase-1 / phase-2 orchestration.
//
// Floating-point statistics that must match the reference bit for bit
// (means, inverse sds, residual variances, HWE thresholds) are computed on
// the host from exact integer code counts produced on the device, with the
// reference's formulas (genotype.cpp:629-689, gwldcore.cpp:3220-3333).
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <limits>
#include <list>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <sys/mman.h>
#include <sys/stat.h>
#include <functional>
#include <thread>
#include <unistd.h>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/lds.h"
#include "lds_device.cuh"
#include "lds_internal.h"
#include "lds_umma.h"

namespace lds {

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

thread_local std::string g_err;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error(code, buf);
}

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(LDS_ERR_CUDA, "CUDA error in %s: %s", what, cudaGetErrorString(e));
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return LDS_OK;
    } catch (const Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return LDS_ERR_INTERNAL;
    }
}

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
// Owning device allocation; move-only so containers never double-free.
// Stream-ordered allocation target of this thread: while a PoolScope is alive,
// DevBuf allocations come from the library's private memory pool on its stream
// and go back to it with cudaFreeAsync, which (unlike cudaFree) does not wait
// for the whole device; the pool keeps its reservation for later calls.
struct PoolTarget {
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
};
thread_local PoolTarget t_pool;

struct PoolScope {
    PoolTarget saved;
    PoolScope(cudaMemPool_t pool, cudaStream_t st) : saved(t_pool) { t_pool = {pool, st}; }
    ~PoolScope() { t_pool = saved; }
};

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    cudaStream_t pool_st = nullptr;  // non-null: pool memory, freed in this stream's order
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), pool_st(o.pool_st) {
        o.p = nullptr;
        o.n = 0;
        o.pool_st = nullptr;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            pool_st = o.pool_st;
            o.p = nullptr;
            o.n = 0;
            o.pool_st = nullptr;
        }
        return *this;
    }
    void* get(size_t bytes) {
        if (bytes <= n && p) return p;
        release();
        if (bytes == 0) bytes = 16;
        if (t_pool.pool) {
            ck(cudaMallocFromPoolAsync(&p, bytes, t_pool.pool, t_pool.st), "pool allocation");
            pool_st = t_pool.st;
        } else {
            ck(cudaMalloc(&p, bytes), "cudaMalloc");
        }
        n = bytes;
        return p;
    }
    template <typename T>
    T* as(size_t count) { return static_cast<T*>(get(count * sizeof(T))); }
    void release() {
        if (p) {
            if (pool_st) cudaFreeAsync(p, pool_st);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
        pool_st = nullptr;
    }
    ~DevBuf() { release(); }
};

template <typename T>
void h2d(T* d, const T* h, size_t count, cudaStream_t st) {
    if (count) ck(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, st), "H2D");
}
template <typename T>
void d2h(T* h, const T* d, size_t count, cudaStream_t st) {
    if (count) ck(cudaMemcpyAsync(h, d, count * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H");
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// 2-D uint8 TMA descriptor over a row-major device buffer (each copy lands in the
// issuing CTA's own shared memory).
CUtensorMap make_map_2d(void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
                        uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swz) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    if (!encode) fail(LDS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    CUtensorMap m;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(LDS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return m;
}

// Phase-2 implementation: 1 = tcgen05 (default; needs 4 digits), 0 = mma.sync.
int& p2_impl() {
    static int v = [] {
        const char* s = std::getenv("LDS_P2_KERNEL");
        return (s && !strcmp(s, "mma")) ? 0 : 1;
    }();
    return v;
}

// ---------------------------------------------------------------------------
// Prepared genotype image + statistics
// ---------------------------------------------------------------------------
struct Prepared {
    std::string key;
    DevGeno g;
    DevBuf codes;
    std::vector<SnpCounts> counts;    // after imputation (HWE) or raw (mean)
    std::vector<double> mean, sdinv;  // per SNP, the reference's formulas
    // 1 for a SNP whose standardized genotypes are identically zero: all
    // calls missing, or every observed (or completed) call the same.  Such a
    // SNP contributes exactly nothing to any product, but the reference's
    // residual-variance weight for it is 1/sqrt(eps) (1e5 at the default
    // eps); left in a phase-1 weight column it would set that column's digit
    // scale and cost every other SNP in the column ~17 bits of precision, so
    // the member lists leave it out.
    std::vector<uint8_t> constant;
    int impute = LDS_IMPUTE_MEAN;
    int ddof = 1;
    DevBuf d_mean, d_sdinv;
    // Per SNP row: 1 when the row has a missing call (after imputation).  When
    // some rows have none (HWE-completed images, fully observed data), phase 2
    // skips the O plane on 128-SNP tiles without missing calls.
    DevBuf d_missing;
    bool has_complete = false;
};

struct Context {
    std::mutex mu;
    bool ready = false;
    int device = -1;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[8];
    unsigned* checked_err = nullptr;  // bounds-checked build: first failed index check
    std::list<std::unique_ptr<Prepared>> cache;  // most recent first
    DevBuf raw, rows_dev, hwe_q0, hwe_q01, hwe_sb, counts_dev, units_dev;
    // Image preparation stream of the streamed one-call windowed estimate
    // (highest priority, so its short kernels are scheduled between the
    // estimate's CTAs), and a grow-only pinned staging area for its results.
    cudaStream_t st_prep = nullptr;
    cudaMemPool_t pool = nullptr;   // chunk images and plans (PoolScope on st_prep)
    void* pinned = nullptr;
    size_t pinned_n = 0;
    DevBuf y, yq, ycs, wq, wcs, z, rowind, sc, binoff, wqoff, accum, mc, guards, lscale, xin;
    DevBuf colsum;  // per-block phase 2: sketch digit column sums (images with complete tiles)
    // Surrogate-network workspace, grow-only so that repeated training and
    // inference calls make no device allocations (cudaFree synchronizes).
    DevBuf mlp_m, mlp_v, mlp_g, mlp_zs, mlp_dzs, mlp_dout, mlp_rows, mlp_loss, mlp_pack;
    // Sketch-digit (0) and weight-digit (1) workspaces shared by windowed plans:
    // grow-only, and each plan keeps the buffer its graph captured alive, so
    // creating and destroying plans does not allocate and free gigabytes.
    std::shared_ptr<DevBuf> ws[2];
    double timings[4] = {0, 0, 0, 0};
    int slices = 4;
    // Non-finite / extreme updates dropped by the last per-block phase 2.
    unsigned long long last_guards[2] = {0, 0};
};

Context& ctx() {
    static Context c;
    return c;
}

void ensure_device(Context& c) {
    if (c.ready) return;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
        fail(LDS_ERR_CUDA, "no CUDA device available (liblds has no CPU fallback)");
    ck(cudaGetDevice(&c.device), "cudaGetDevice");
    ck(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : c.ev) ck(cudaEventCreate(&e), "cudaEventCreate");
#ifdef LDS_CHECKED
    // The bounds-checked build's device error word, published to every file's
    // copy of the pointer.
    ck(cudaMalloc(&c.checked_err, sizeof(unsigned)), "checked error word");
    ck(cudaMemset(c.checked_err, 0, sizeof(unsigned)), "checked error word");
    for (CheckedErrSetter f : checked_err_setters()) ck(f(c.checked_err), "checked error word");
#endif
    c.ready = true;
}

// Mean and inverse sd over observed calls (genotype.cpp:651-689).
void stats_observed(long long nobs, long long sum, long long sumsq, int ddof, double& mu,
                    double& inv_sd) {
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

// Mean and inverse sd after completion (genotype.cpp:629-649).
void stats_completed(long long sum, long long sumsq, int n, int ddof, double& mean,
                     double& inv_std) {
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

uint64_t hwe_seed_base(uint64_t impute_seed, int global_snp) {
    uint64_t h = mix64(impute_seed);
    h ^= mix64((uint64_t)(uint32_t)global_snp + 0x243f6a8885a308d3ULL);
    return h;
}

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ULL) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// Upload raw SNP-major rows, repack, count, impute, and compute statistics.
// `global_snp0` is the genome index of the first row (HWE seeds use it).
// Seeded synthetic genotypes generated straight into the image (no host copy).
struct SynthSpec {
    uint64_t seed;
    const int64_t* t0;  // host, M thresholds each
    const int64_t* t1;
    int missing;
};

std::unique_ptr<Prepared> prepare(Context& c, const uint8_t* host_rows, int64_t row_bytes,
                                  int64_t n_total, int64_t M, const int64_t* row_sel,
                                  int64_t n_sel, int impute, uint64_t impute_seed, int ddof,
                                  const std::string& key, const SynthSpec* synth = nullptr,
                                  int64_t snp_base = 0) {
    auto P = std::make_unique<Prepared>();
    P->key = key;
    P->impute = impute;
    P->ddof = ddof;
    DevGeno& g = P->g;
    g.N = row_sel ? n_sel : n_total;
    if (g.N <= 0) fail(LDS_ERR_ARG, "no samples selected");
    g.N_pad = round_up(g.N, kSamplePad);
    g.nbp = g.N_pad / 4;
    g.M = M;
    g.M_pad = round_up(std::max<int64_t>(M, 1), kSnpPad) + kSnpPad;
    g.codes = P->codes.as<uint8_t>((size_t)(g.M_pad * g.nbp));

    std::vector<int32_t> rows32;
    int32_t* d_rows = nullptr;
    if (row_sel) {
        rows32.resize((size_t)n_sel);
        for (int64_t i = 0; i < n_sel; ++i) {
            if (row_sel[i] < 0 || row_sel[i] >= n_total)
                fail(LDS_ERR_ARG, "row_sel contains an out-of-range sample index");
            rows32[(size_t)i] = (int32_t)row_sel[i];
        }
        d_rows = c.rows_dev.as<int32_t>(rows32.size());
        h2d(d_rows, rows32.data(), rows32.size(), c.st);
    }
    if (synth) {
        if (row_sel) fail(LDS_ERR_ARG, "synthetic images take no sample selection");
        DevBuf dt0, dt1;
        int64_t* a = dt0.as<int64_t>((size_t)std::max<int64_t>(M, 1));
        int64_t* b = dt1.as<int64_t>((size_t)std::max<int64_t>(M, 1));
        h2d(a, synth->t0, (size_t)M, c.st);
        h2d(b, synth->t1, (size_t)M, c.st);
        launch_synth(n_total, M, synth->seed, a, b, synth->missing, g.codes, c.st, g.nbp, 1);
        ck(cudaStreamSynchronize(c.st), "synthetic image");
    }
    // Upload in slabs to bound the staging buffer.
    const int64_t slab_rows =
        std::max<int64_t>(1, std::min<int64_t>(M, (int64_t)(1LL << 30) / std::max<int64_t>(row_bytes, 1)));
    uint8_t* d_raw = synth ? nullptr : c.raw.as<uint8_t>((size_t)(slab_rows * row_bytes));
    for (int64_t j0 = 0; !synth && j0 < M; j0 += slab_rows) {
        const int64_t nr = std::min(slab_rows, M - j0);
        h2d(d_raw, host_rows + j0 * row_bytes, (size_t)(nr * row_bytes), c.st);
        DevGeno sub = g;
        sub.M = nr;
        sub.M_pad = nr;
        sub.codes = g.codes + j0 * g.nbp;
        launch_repack(d_raw, row_bytes, n_total, d_rows, sub, c.st);
    }
    // Padding rows (all code 01).
    if (g.M_pad > M)
        ck(cudaMemsetAsync(g.codes + M * g.nbp, 0x55, (size_t)((g.M_pad - M) * g.nbp), c.st),
           "memset pad rows");

    SnpCounts* d_counts = c.counts_dev.as<SnpCounts>((size_t)std::max<int64_t>(M, 1));
    P->counts.resize((size_t)M);
    launch_counts(g, d_counts, c.st);
    d2h(P->counts.data(), d_counts, (size_t)M, c.st);
    ck(cudaStreamSynchronize(c.st), "counts");

    P->mean.resize((size_t)M);
    P->sdinv.resize((size_t)M);
    if (impute == LDS_IMPUTE_HWE) {
        std::vector<double> q0((size_t)M), q01((size_t)M);
        std::vector<uint64_t> sb((size_t)M);
        bool any_missing = false;
        for (int64_t j = 0; j < M; ++j) {
            const SnpCounts& k = P->counts[(size_t)j];
            const long long nobs = (long long)k.n[0] + k.n[1] + k.n[2];
            const long long sum = (long long)k.n[1] + 2LL * k.n[2];
            double p = 0.0;
            if (nobs > 0) {
                p = (double)sum / (2.0 * (double)nobs);
                if (p < 0.0) p = 0.0;
                if (p > 1.0) p = 1.0;
            }
            q0[(size_t)j] = (1.0 - p) * (1.0 - p);
            q01[(size_t)j] = q0[(size_t)j] + 2.0 * p * (1.0 - p);
            sb[(size_t)j] = hwe_seed_base(impute_seed, (int)(snp_base + j));
            any_missing |= k.n[3] > 0;
        }
        if (any_missing) {
            double* dq0 = c.hwe_q0.as<double>((size_t)M);
            double* dq01 = c.hwe_q01.as<double>((size_t)M);
            uint64_t* dsb = c.hwe_sb.as<uint64_t>((size_t)M);
            h2d(dq0, q0.data(), (size_t)M, c.st);
            h2d(dq01, q01.data(), (size_t)M, c.st);
            h2d(dsb, sb.data(), (size_t)M, c.st);
            launch_hwe_impute(g, dq0, dq01, dsb, d_rows, c.st);
            launch_counts(g, d_counts, c.st);
            d2h(P->counts.data(), d_counts, (size_t)M, c.st);
            ck(cudaStreamSynchronize(c.st), "hwe counts");
        }
        for (int64_t j = 0; j < M; ++j) {
            const SnpCounts& k = P->counts[(size_t)j];
            const long long sum = (long long)k.n[1] + 2LL * k.n[2];
            const long long sumsq = (long long)k.n[1] + 4LL * k.n[2];
            stats_completed(sum, sumsq, (int)g.N, ddof, P->mean[(size_t)j], P->sdinv[(size_t)j]);
        }
    } else {
        for (int64_t j = 0; j < M; ++j) {
            const SnpCounts& k = P->counts[(size_t)j];
            const long long nobs = (long long)k.n[0] + k.n[1] + k.n[2];
            const long long sum = (long long)k.n[1] + 2LL * k.n[2];
            const long long sumsq = (long long)k.n[1] + 4LL * k.n[2];
            stats_observed(nobs, sum, sumsq, ddof, P->mean[(size_t)j], P->sdinv[(size_t)j]);
        }
    }
    P->constant.resize((size_t)M);
    std::vector<uint8_t> miss((size_t)M);
    for (int64_t j = 0; j < M; ++j) {
        const SnpCounts& k = P->counts[(size_t)j];
        const int classes = (k.n[0] > 0) + (k.n[1] > 0) + (k.n[2] > 0);
        P->constant[(size_t)j] = classes <= 1 ? 1 : 0;
        miss[(size_t)j] = k.n[3] > 0 ? 1 : 0;
        if (!miss[(size_t)j]) P->has_complete = true;
    }
    h2d(P->d_missing.as<uint8_t>((size_t)std::max<int64_t>(M, 1)), miss.data(), (size_t)M, c.st);
    double* dm = P->d_mean.as<double>((size_t)std::max<int64_t>(M, 1));
    double* ds = P->d_sdinv.as<double>((size_t)std::max<int64_t>(M, 1));
    h2d(dm, P->mean.data(), (size_t)M, c.st);
    h2d(ds, P->sdinv.data(), (size_t)M, c.st);
    ck(cudaStreamSynchronize(c.st), "prepare");
    return P;
}

// Sum of squared standardized values of SNP j, from code counts; values are
// rounded to T first like the reference's standardized block
// (gwldcore.cpp:3275-3284 sums x^2 of the T-typed block).
template <typename T>
double sumsq_std(const Prepared& P, int64_t j) {
    const SnpCounts& k = P.counts[(size_t)j];
    const double mu = P.mean[(size_t)j], s = P.sdinv[(size_t)j];
    double acc = 0.0;
    for (int c = 0; c < 3; ++c) {
        const double x = (double)(T)(((double)c - mu) * s);
        acc += (double)k.n[c] * (x * x);
    }
    return acc;
}

// inv_j = 1/sqrt(max(eps, ||x_j||^2/(N-1))) (gwldcore.cpp:3320-3331).
template <typename T>
T inv_resvar(const Prepared& P, int64_t j, double eps) {
    const double var = sumsq_std<T>(P, j) / (double)(P.g.N - 1);
    const double safe = std::isnan(var) ? var : (var > eps ? var : eps);
    return (T)(1.0 / std::sqrt(safe));
}

// ---------------------------------------------------------------------------
// Probe streams: mt19937_64 seeded per (root, block start, V-tile start)
// (gwldcore.cpp:452-458, :1691-1716).  Column-major L x V into Z (ld = z_ld).
// ---------------------------------------------------------------------------
uint64_t probe_seed(uint64_t root, int blk_start, int v_start) {
    uint64_t s = 0x1234abcdULL;
    s ^= mix64(root);
    s ^= mix64((uint64_t)blk_start + 0x9e37ULL);
    s ^= mix64((uint64_t)v_start + 0x85ebULL);
    return s;
}

template <typename T>
void make_probes(uint64_t root, int blk_start, int v_start, int L, int V, int dist, double* Z,
                 int64_t z_ld) {
    std::mt19937_64 rng(probe_seed(root, blk_start, v_start));
    std::normal_distribution<T> gN(0, (T)1);
    std::vector<T> col((size_t)L);
    for (int c = 0; c < V; ++c) {
        long double ss = 0.0L;
        for (int r = 0; r < L; ++r) {
            const T z = (dist == LDS_DIST_RADEMACHER) ? ((rng() & 1) ? T(1) : T(-1)) : gN(rng);
            col[(size_t)r] = z;
            if (dist == LDS_DIST_SPHERICAL) ss += (long double)z * (long double)z;
        }
        if (dist == LDS_DIST_SPHERICAL) {
            const T zs = ss > 0.0L ? (T)std::sqrt((long double)L / ss) : T(1);
            for (int r = 0; r < L; ++r) col[(size_t)r] *= zs;
        }
        for (int r = 0; r < L; ++r) Z[(int64_t)c * z_ld + r] = (double)col[(size_t)r];
    }
}

// Rademacher probe blocks generated on the device (lds_probes.cu): the same
// mt19937_64 streams as make_probes, written straight into dZ.
void device_rademacher(Context& c, const std::vector<ProbeUnit>& units, int V, double* dZ,
                       int64_t ld) {
    if (units.empty()) return;
    // The unit table lives in a grow-only context buffer: no cudaFree (which
    // waits for the whole device) while other streams are busy.
    ProbeUnit* d = c.units_dev.as<ProbeUnit>(units.size());
    h2d(d, units.data(), units.size(), c.st);
    launch_rademacher_units(d, (int64_t)units.size(), V, dZ, ld, c.st);
    ck(cudaGetLastError(), "probe streams");
    ck(cudaStreamSynchronize(c.st), "probe streams");  // the table is reused by the next call
}

// ---------------------------------------------------------------------------
// Phase-1 CSR over annotation bins (build_phase1_csr, gwldcore.cpp:1002-1063).
// annot: L x K row-major (values as T), inv: L (as T); SNP j = snp0 + i.
// ---------------------------------------------------------------------------
struct Csr {
    std::vector<int64_t> bin_off;   // K+1, padded to kSnpStep
    std::vector<int32_t> rowind;
    std::vector<double> sc;
    std::vector<int64_t> nnz;       // real members per bin
    std::vector<int64_t> wq_off;    // K, bytes
    int64_t wq_bytes = 0;
};

template <typename T>
Csr build_csr(const T* annot, const T* inv, int64_t L, int64_t K, int64_t snp0, int Vp, int S,
              int64_t pad = kSnpStep, const uint8_t* constant = nullptr) {
    Csr c;
    c.bin_off.assign((size_t)K + 1, 0);
    c.nnz.assign((size_t)K, 0);
    c.wq_off.assign((size_t)K, 0);
    std::vector<std::vector<std::pair<int32_t, double>>> members((size_t)K);
    for (int64_t k = 0; k < K; ++k) {
        for (int64_t i = 0; i < L; ++i) {
            const T a = annot[i * K + k];
            if (a == T(0)) continue;
            if (constant && constant[snp0 + i]) continue;  // contributes exactly zero
            const double ad = (double)a;
            if (!(ad > 0.0) || !std::isfinite(ad)) continue;
            const double invd = (double)inv[i];
            if (!std::isfinite(invd) || invd <= 0.0) continue;
            const double s = invd * std::sqrt(ad);
            if (!std::isfinite(s)) continue;
            if (std::is_same<T, float>::value && s > (double)std::numeric_limits<float>::max())
                continue;
            members[(size_t)k].push_back({(int32_t)(snp0 + i), (double)(T)s});
        }
    }
    int64_t off = 0, wq = 0;
    for (int64_t k = 0; k < K; ++k) {
        const int64_t n = (int64_t)members[(size_t)k].size();
        const int64_t np = round_up(n, pad);
        c.nnz[(size_t)k] = n;
        c.bin_off[(size_t)k] = off;
        c.wq_off[(size_t)k] = wq;
        off += np;
        wq += (int64_t)S * 2 * Vp * np;
    }
    c.bin_off[(size_t)K] = off;
    c.wq_bytes = wq;
    c.rowind.assign((size_t)off, (int32_t)snp0);
    c.sc.assign((size_t)off, 0.0);
    for (int64_t k = 0; k < K; ++k) {
        int64_t p = c.bin_off[(size_t)k];
        for (auto& m : members[(size_t)k]) {
            c.rowind[(size_t)p] = m.first;
            c.sc[(size_t)p] = m.second;
            ++p;
        }
    }
    return c;
}

// Run phase 1 for all bins of `csr` with probes Z (rows z_row0.., ld z_ld),
// leaving Y (N_pad x K*V FP64) in c.y.
void run_phase1(Context& c, Prepared& P, const Csr& csr, int64_t K, int V, const double* Z_host,
                int64_t z_ld, int64_t z_rows, int64_t z_row0) {
    const int S = c.slices;
    const int Vp = (int)round_up(V, kColTile);
    const int64_t nm = std::max<int64_t>((int64_t)csr.rowind.size(), 1);
    int32_t* d_rowind = c.rowind.as<int32_t>((size_t)nm);
    double* d_sc = c.sc.as<double>((size_t)nm);
    int64_t* d_binoff = c.binoff.as<int64_t>(csr.bin_off.size());
    int64_t* d_wqoff = c.wqoff.as<int64_t>(std::max<size_t>(csr.wq_off.size(), 1));
    h2d(d_rowind, csr.rowind.data(), csr.rowind.size(), c.st);
    h2d(d_sc, csr.sc.data(), csr.sc.size(), c.st);
    h2d(d_binoff, csr.bin_off.data(), csr.bin_off.size(), c.st);
    h2d(d_wqoff, csr.wq_off.data(), csr.wq_off.size(), c.st);
    double* d_z = c.z.as<double>((size_t)std::max<int64_t>(z_ld * V, 1));
    h2d(d_z, Z_host, (size_t)(z_ld * V), c.st);
    (void)z_rows;

    P1Weights w;
    w.K = (int)K;
    w.V = V;
    w.Vp = Vp;
    w.S = S;
    w.rowind = d_rowind;
    w.sc = d_sc;
    w.bin_off = d_binoff;
    w.wq_off = d_wqoff;
    w.wq = c.wq.as<int8_t>((size_t)std::max<int64_t>(csr.wq_bytes, 16));
    w.colscale = c.wcs.as<double>((size_t)(K * Vp));
    launch_p1_weights(w, static_cast<double*>(P.d_mean.p), static_cast<double*>(P.d_sdinv.p), d_z,
                      z_ld, z_row0, c.st);
    double* Y = c.y.as<double>((size_t)(P.g.N_pad * K * V));
    launch_p1(P.g, w, csr.bin_off.data(), Y, c.st);
}

// The per-block phase 2 runs on the tcgen05 kernel (lds_umma.cu) with the
// default 4 digits; other digit counts, or the mma.sync kernel selected for
// cross-checks (lds_set_p2_kernel), use the warp-level kernel.
bool per_block_umma(const Context& c) { return c.slices == 4 && p2_impl() == 1; }

// Quantize the device sketch in c.y (N_pad x K*V) into c.yq.
void quantize_sketch(Context& c, Prepared& P, int64_t K, int V) {
    if (per_block_umma(c)) {
        const int nc = umma::ncolp_for(V);
        int8_t* yq = c.yq.as<int8_t>((size_t)(K * nc * P.g.N_pad));
        double* cs = c.ycs.as<double>((size_t)(K * V));
        int* colsum = P.has_complete ? c.colsum.as<int>((size_t)(K * nc)) : nullptr;
        umma::launch_quantize_y4(static_cast<double*>(c.y.p), P.g.N, P.g.N_pad, (int)K, V, nc, yq,
                                 cs, c.st, colsum);
        return;
    }
    const int S = c.slices;
    const int Vp = (int)round_up(V, kColTile);
    int8_t* yq = c.yq.as<int8_t>((size_t)(S * K * Vp * P.g.N_pad));
    double* cs = c.ycs.as<double>((size_t)(K * Vp));
    launch_quantize_y(static_cast<double*>(c.y.p), P.g.N, P.g.N_pad, (int)K, V, Vp, S, yq, cs,
                      c.st);
}

// Phase 2 over SNPs [j0, j1) into device accumulators (out_row0 offset).
double extreme_warn_env() {
    static const double warn = [] {
        const char* s = std::getenv("SUMMIT_P2_EXTREME_LD_WARN");
        if (!s || !*s) s = std::getenv("SUMMIT_P2_ABS_LD_MAX");
        double v = 1.0e10;
        if (s && *s) {
            char* end = nullptr;
            const double x = std::strtod(s, &end);
            if (end != s && std::isfinite(x)) v = x;
        }
        return v > 0.0 ? v : std::numeric_limits<double>::infinity();
    }();
    return warn;
}

int drop_extreme_env() {
    static const int drop = [] {
        const char* s = std::getenv("SUMMIT_P2_DROP_EXTREME");
        if (!s || !*s) return 1;
        if (!strcmp(s, "0") || !strcmp(s, "false") || !strcmp(s, "FALSE") || !strcmp(s, "no") ||
            !strcmp(s, "NO"))
            return 0;
        return 1;
    }();
    return drop;
}

void run_phase2(Context& c, Prepared& P, int64_t K, int V, int64_t j0, int64_t j1,
                int64_t out_row0, double* d_accum, double* d_mc, const double* d_lscale) {
    // c.guards: [0] non-finite drops, [1] extreme drops, [2] kernel status
    // (zeroed by the caller before each call).
    unsigned long long* guards = c.guards.as<unsigned long long>(4);
    if (per_block_umma(c)) {
        const int nc = umma::ncolp_for(V);
        umma::P2UArgs u;
        u.K = (int)K;
        u.V = V;
        u.ncolp = nc;
        u.bins_per_cta = umma::p2_bins_per_cta(nc, (int)K);
        u.ngroups = (u.bins_per_cta * nc + 255) / 256;
        u.box_rows = std::min(256, u.bins_per_cta * nc);
        u.nkt = (int)(P.g.N_pad / 128);
        u.M = P.g.M;
        u.j0 = j0;
        u.j1 = j1;
        u.out_row0 = out_row0;
        u.colscale = static_cast<double*>(c.ycs.p);
        u.mean = static_cast<double*>(P.d_mean.p);
        u.sdinv = static_cast<double*>(P.d_sdinv.p);
        u.left_scale = d_lscale;
        u.accum = d_accum;
        u.mc = d_mc;
        u.guard_counts = guards;
        u.extreme_warn = extreme_warn_env();
        u.drop_extreme = drop_extreme_env();
        u.status = reinterpret_cast<unsigned*>(guards + 2);
        if (P.has_complete) {
            u.snp_missing = static_cast<const uint8_t*>(P.d_missing.p);
            u.colsum = static_cast<const int*>(c.colsum.p);
        }
        const CUtensorMap tA = make_map_2d(P.g.codes, (uint64_t)P.g.nbp, (uint64_t)P.g.M_pad,
                                           (uint64_t)P.g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
        u.yq = static_cast<const int8_t*>(c.yq.p);
        u.yq_cols = K * nc;
        umma::launch_p2_umma(tA, u, c.st);
        return;
    }
    P2Args a;
    a.K = (int)K;
    a.V = V;
    a.Vp = (int)round_up(V, kColTile);
    a.S = c.slices;
    a.j0 = j0;
    a.j1 = j1;
    a.out_row0 = out_row0;
    a.Yq = static_cast<int8_t*>(c.yq.p);
    a.colscale = static_cast<double*>(c.ycs.p);
    a.mean = static_cast<double*>(P.d_mean.p);
    a.sdinv = static_cast<double*>(P.d_sdinv.p);
    a.left_scale = d_lscale;
    a.accum = d_accum;
    a.mc = d_mc;
    a.guard_counts = guards;
    a.extreme_warn = extreme_warn_env();
    a.drop_extreme = drop_extreme_env();
    launch_p2(P.g, a, c.st);
}

void report_guards(Context& c, const char* label, int blk_start, int blk_end) {
    unsigned long long h[3] = {0, 0, 0};
    d2h(h, static_cast<unsigned long long*>(c.guards.p), 3, c.st);
    ck(cudaStreamSynchronize(c.st), "guards");
    c.last_guards[0] = h[0];
    c.last_guards[1] = h[1];
    if ((unsigned)h[2] != 0)
        fail(LDS_ERR_CUDA, "phase-2 kernel aborted in %s block [%d:%d): a pipeline wait ran out "
             "(status %u)", label, blk_start, blk_end, (unsigned)h[2]);
    if (h[0])
        std::fprintf(stderr,
                     "[phase2-warning] %s block [%d:%d): dropped %llu non-finite LD-score updates.\n",
                     label, blk_start, blk_end, h[0]);
    if (h[1])
        std::fprintf(stderr,
                     "[phase2-warning] %s block [%d:%d): %llu finite updates exceeded the "
                     "LD-score warning threshold. They were dropped unless "
                     "SUMMIT_P2_DROP_EXTREME=0; inspect this run before using it.\n",
                     label, blk_start, blk_end, h[1]);
}

// ---------------------------------------------------------------------------
// Files: identity key, FAM/BIM line counts, mapped BED.
// ---------------------------------------------------------------------------
std::string file_identity(const std::string& path) {
    struct stat s {};
    if (::stat(path.c_str(), &s) != 0) fail(LDS_ERR_IO, "Failed to stat input path: %s", path.c_str());
    char buf[512];
    snprintf(buf, sizeof buf, "%s#%llu:%llu:%llu:%lld.%ld:%lld.%ld", path.c_str(),
             (unsigned long long)s.st_dev, (unsigned long long)s.st_ino,
             (unsigned long long)s.st_size, (long long)s.st_mtim.tv_sec, s.st_mtim.tv_nsec,
             (long long)s.st_ctim.tv_sec, s.st_ctim.tv_nsec);
    return buf;
}

int64_t count_lines(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) fail(LDS_ERR_IO, "Failed to open file: %s", path.c_str());
    int64_t n = 0;
    char* line = nullptr;
    size_t cap = 0;
    ssize_t len;
    while ((len = getline(&line, &cap, f)) != -1) {
        if (len > 0 && line[0] == '#') continue;
        ++n;
    }
    std::free(line);
    std::fclose(f);
    return n;
}

struct MappedBed {
    int fd = -1;
    size_t size = 0;
    uint8_t* base = nullptr;
    explicit MappedBed(const std::string& path) {
        fd = ::open(path.c_str(), O_RDONLY | O_CLOEXEC);
        if (fd < 0) fail(LDS_ERR_IO, "Failed to open bed: %s", path.c_str());
        struct stat st {};
        if (::fstat(fd, &st) != 0 || st.st_size < 3)
            fail(LDS_ERR_IO, "stat failed or BED too small: %s", path.c_str());
        size = (size_t)st.st_size;
        void* p = ::mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) fail(LDS_ERR_IO, "mmap failed for: %s", path.c_str());
        base = static_cast<uint8_t*>(p);
        if (!(base[0] == 0x6C && base[1] == 0x1B && base[2] == 0x01))
            fail(LDS_ERR_IO, "Invalid BED magic/mode (expected 6C 1B 01) for: %s", path.c_str());
    }
    ~MappedBed() {
        if (base) ::munmap(base, size);
        if (fd >= 0) ::close(fd);
    }
};

std::string sel_key(const int64_t* rows, int64_t n) {
    if (!rows) return "all";
    char b[64];
    snprintf(b, sizeof b, "%lld:%016llx", (long long)n,
             (unsigned long long)fnv1a(rows, (size_t)n * sizeof(int64_t)));
    return b;
}

// Device image of a BED fileset, cached by file identity, sample selection,
// imputation mode/seed and ddof (like the reference's mapping cache,
// genotype.cpp:350-410, keyed by file identity).
Prepared& prepared_for_file(Context& c, const std::string& bed_prefix, const std::string& fam,
                            const int64_t* rows, int64_t n_rows, int impute, uint64_t iseed,
                            int ddof, int64_t* M_total_out) {
    const std::string bed = bed_prefix + ".bed";
    const std::string bim = bed_prefix + ".bim";
    const int64_t n_total = count_lines(fam);
    if (n_total <= 0) fail(LDS_ERR_IO, "FAM has zero rows: %s", fam.c_str());
    const int64_t M = count_lines(bim);
    if (M_total_out) *M_total_out = M;
    char kb[128];
    snprintf(kb, sizeof kb, "|%d|%llu|%d|%lld", impute,
             (unsigned long long)(impute == LDS_IMPUTE_HWE ? iseed : 0ULL), ddof, (long long)n_total);
    const std::string key = file_identity(bed) + "|" + sel_key(rows, n_rows) + kb;
    for (auto it = c.cache.begin(); it != c.cache.end(); ++it) {
        if ((*it)->key == key) {
            c.cache.splice(c.cache.begin(), c.cache, it);
            return *c.cache.front();
        }
    }
    MappedBed mb(bed);
    const int64_t nbytes = (n_total + 3) / 4;
    if ((size_t)(3 + M * nbytes) > mb.size)
        fail(LDS_ERR_IO, "BED file too small for requested block: %s", bed.c_str());
    while (c.cache.size() >= 2) c.cache.pop_back();
    auto P = prepare(c, mb.base + 3, nbytes, n_total, M, rows, n_rows, impute, iseed, ddof, key);
    c.cache.push_front(std::move(P));
    return *c.cache.front();
}

// Exact-digit products x_j . y_v of the standardized genotypes of SNPs [j0, j1)
// with the columns of a dense N x V matrix Y (column-major, FP64): the phase-2
// tensor-core kernel in its raw-product mode (G^T y and O^T y per digit set,
// recombined exactly), then x_j . y = s_j colscale_v (G^T y - mu_j O^T y).
// Returns (j1 - j0) x V row-major.
std::vector<double> snp_products(Context& c, const Prepared& P, int64_t j0, int64_t j1,
                                 const std::vector<double>& Y, int64_t V) {
    const int64_t L = j1 - j0, N = P.g.N, Np = P.g.N_pad;
    std::vector<double> out((size_t)(L * V), 0.0);
    if (L <= 0 || V <= 0) return out;
    if (c.slices != 4 || p2_impl() != 1)
        fail(LDS_ERR_ARG, "covariate products need the tcgen05 kernels with 4 digits");
    std::vector<double> y((size_t)(Np * V), 0.0);
    for (int64_t v = 0; v < V; ++v)
        std::memcpy(&y[(size_t)(v * Np)], &Y[(size_t)(v * N)], sizeof(double) * (size_t)N);
    DevBuf dy, dyq, dcs, rg, ro, st;
    double* d_y = dy.as<double>(y.size());
    h2d(d_y, y.data(), y.size(), c.st);
    const int nc = umma::ncolp_for((int)V);
    int8_t* yq = dyq.as<int8_t>((size_t)(nc * Np));
    double* cs = dcs.as<double>((size_t)V);
    umma::launch_quantize_y4(d_y, N, Np, 1, (int)V, nc, yq, cs, c.st);
    long long* dg = rg.as<long long>((size_t)(L * V));
    long long* dO = ro.as<long long>((size_t)(L * V));
    unsigned* dst = st.as<unsigned>(1);
    ck(cudaMemsetAsync(dst, 0, 4, c.st), "memset");
    const CUtensorMap tA = make_map_2d(P.g.codes, (uint64_t)P.g.nbp, (uint64_t)P.g.M_pad,
                                       (uint64_t)P.g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
    umma::P2UArgs u;
    u.yq = yq;
    u.yq_cols = nc;
    u.K = 1;
    u.V = (int)V;
    u.ncolp = nc;
    u.ngroups = (nc + 255) / 256;
    u.box_rows = std::min(256, nc);
    u.nkt = (int)(Np / 128);
    u.M = P.g.M;
    u.j0 = j0;
    u.j1 = j1;
    u.out_row0 = j0;
    u.colscale = cs;
    u.mean = static_cast<double*>(P.d_mean.p);
    u.sdinv = static_cast<double*>(P.d_sdinv.p);
    u.status = dst;
    u.raw_g = dg;
    u.raw_o = dO;
    umma::launch_p2_umma(tA, u, c.st);
    ck(cudaGetLastError(), "launch");
    std::vector<long long> hg((size_t)(L * V)), ho((size_t)(L * V));
    std::vector<double> hcs((size_t)V);
    unsigned stv = 0;
    d2h(hg.data(), dg, hg.size(), c.st);
    d2h(ho.data(), dO, ho.size(), c.st);
    d2h(hcs.data(), cs, hcs.size(), c.st);
    d2h(&stv, dst, 1, c.st);
    ck(cudaStreamSynchronize(c.st), "snp products");
    if (stv) fail(LDS_ERR_CUDA, "phase-2 tensor-core pipeline wait timed out (code %u)", stv);
    for (int64_t j = 0; j < L; ++j) {
        const double mu = P.mean[(size_t)(j0 + j)], sd = P.sdinv[(size_t)(j0 + j)];
        for (int64_t v = 0; v < V; ++v) {
            const size_t q = (size_t)(j * V + v);
            out[q] = sd * hcs[(size_t)v] * ((double)hg[q] - mu * (double)ho[q]);
        }
    }
    return out;
}

// Residual variances with covariates, fused form (compute_inv_resvar_from_geno_block,
// gwldcore.cpp:3220-3333): ss_j = ||x_j||^2 + q - 2h with proj = R x_j,
// h = ||proj||^2, q = proj^T G proj (G = resvar_gram, row-major p x p) or h;
// df = N - p - 1.
template <typename T>
void inv_resvar_fused_cov(Context& c, const Prepared& P, int64_t j0, int64_t L, const T* Cm,
                          const T* Rm, int64_t p, const T* gram, double eps, T* inv_out) {
    const int64_t N = P.g.N;
    if ((Cm != nullptr) != (Rm != nullptr))
        fail(LDS_ERR_ARG, "C and R must be provided together for fused residual variances");
    if (N - p <= 1) fail(LDS_ERR_ARG, "N_eff must be > 1 in fused residual variances");
    const double df = (double)(N - p - 1);
    std::vector<double> Rt((size_t)(N * p));
    for (int64_t a = 0; a < p; ++a)
        for (int64_t i = 0; i < N; ++i) Rt[(size_t)(a * N + i)] = (double)Rm[a + i * p];
    const std::vector<double> proj = snp_products(c, P, j0, j0 + L, Rt, p);
    for (int64_t j = 0; j < L; ++j) {
        const double* pr = &proj[(size_t)(j * p)];
        double h = 0.0;
        for (int64_t a = 0; a < p; ++a) h += (double)(T)pr[a] * (double)(T)pr[a];
        double q = h;
        if (gram) {
            q = 0.0;
            for (int64_t a = 0; a < p; ++a) {
                double gy = 0.0;
                for (int64_t b = 0; b < p; ++b) gy += (double)gram[a * p + b] * (double)(T)pr[b];
                q += (double)(T)pr[a] * gy;
            }
        }
        const double ss = sumsq_std<T>(P, j0 + j) + q - 2.0 * h;
        const double var = ss / df;
        const double safe = std::isnan(var) ? var : (var > eps ? var : eps);
        inv_out[j] = (T)(1.0 / std::sqrt(safe));
    }
}

// Residual variances with covariates, block-projection form
// (precompute_residual_variances_bed_impl, gwldcore.cpp:3335-3566):
// ss_j = ||(I - C R) x_j||^2 = ||x||^2 - 2 (C^T x).(R x) + (R x)^T (C^T C) (R x),
// df = N - p - 1; snp_var[j] = min(1, ss / ||x||^2) when requested.
template <typename T>
void inv_resvar_projected_cov(Context& c, const Prepared& P, int64_t nsnps, const T* Cm,
                              const T* Rm, int64_t p, double eps, T* inv_out, double* snp_var) {
    const int64_t N = P.g.N;
    const double df = (double)(N - p - 1);
    if (df <= 0.0) fail(LDS_ERR_ARG, "Projected residual df must be > 0 in precompute_residual_variances_bed");
    std::vector<double> Y((size_t)(N * 2 * p));
    for (int64_t a = 0; a < p; ++a)
        for (int64_t i = 0; i < N; ++i) {
            Y[(size_t)(a * N + i)] = (double)Rm[a + i * p];            // R rows
            Y[(size_t)((p + a) * N + i)] = (double)Cm[a * N + i];      // C columns
        }
    std::vector<double> CtC((size_t)(p * p), 0.0);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) {
            double s = 0.0;
            for (int64_t i = 0; i < N; ++i) s += (double)Cm[a * N + i] * (double)Cm[b * N + i];
            CtC[(size_t)(a * p + b)] = s;
        }
    const int64_t chunk = 1 << 16;
    for (int64_t j0 = 0; j0 < nsnps; j0 += chunk) {
        const int64_t j1 = std::min(nsnps, j0 + chunk);
        const std::vector<double> pr = snp_products(c, P, j0, j1, Y, 2 * p);
        for (int64_t j = j0; j < j1; ++j) {
            const double* rx = &pr[(size_t)((j - j0) * 2 * p)];
            const double* cx = rx + p;
            double cross = 0.0, quad = 0.0;
            for (int64_t a = 0; a < p; ++a) {
                cross += cx[a] * rx[a];
                double gy = 0.0;
                for (int64_t b = 0; b < p; ++b) gy += CtC[(size_t)(a * p + b)] * rx[b];
                quad += rx[a] * gy;
            }
            const double raw = sumsq_std<T>(P, j);
            double ss = raw - 2.0 * cross + quad;
            if (ss < 0.0) ss = 0.0;
            const double var = ss / df;
            const double safe = std::isnan(var) ? var : (var > eps ? var : eps);
            inv_out[j] = (T)(1.0 / std::sqrt(safe));
            if (snp_var) snp_var[j] = (raw > 0.0 && std::isfinite(ss)) ? std::min(1.0, ss / raw) : 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// Entry-point implementations
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Dense genotype blocks, covariate projections inside phase 1 / phase 2, GRM
// panel products, mu22 moments and block corrections
// (gwldcore.cpp:1896-1923, :2602-2649, :2132-2327, :1134-1497, :3335-3627).
// ---------------------------------------------------------------------------
struct DevCov {
    DevBuf C, R;  // FP64, column-major N x p and p x N
    int64_t N = 0, p = 0;
    bool on() const { return p > 0; }
};

template <typename T>
void upload_cov(Context& c, DevCov& d, const T* Cm, const T* Rm, int64_t N, int64_t p) {
    d.N = N;
    d.p = (Cm && Rm) ? p : 0;
    if (!d.on()) return;
    std::vector<double> h((size_t)(N * p));
    for (size_t i = 0; i < h.size(); ++i) h[i] = (double)Cm[i];
    h2d(d.C.as<double>(h.size()), h.data(), h.size(), c.st);
    for (size_t i = 0; i < h.size(); ++i) h[i] = (double)Rm[i];
    h2d(d.R.as<double>(h.size()), h.data(), h.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "covariates");
}

// X (N rows of an ld-strided column-major panel, L columns) <- X - C (R X),
// or with `transpose` X <- X - R^T (C^T X) (the same projection applied from
// the other side).  tmp: p x L scratch.
void project_cols(Context& c, double* X, int64_t ld, int64_t L, const DevCov& cv, bool transpose,
                  DevBuf& tmp) {
    if (!cv.on() || L <= 0) return;
    const int64_t N = cv.N, p = cv.p;
    double* t = tmp.as<double>((size_t)(p * L));
    DGemmArgs a;
    a.M = p;
    a.N = L;
    a.K = N;
    if (transpose) {
        a.A = static_cast<const double*>(cv.C.p);  // C^T: (a, n) -> C[n + a N]
        a.a_ms = N;
        a.a_ks = 1;
    } else {
        a.A = static_cast<const double*>(cv.R.p);  // R: (a, n) -> R[a + n p]
        a.a_ms = 1;
        a.a_ks = p;
    }
    a.B = X;
    a.b_ks = 1;
    a.b_ns = ld;
    a.C = t;
    a.c_ms = 1;
    a.c_ns = p;
    launch_dgemm(a, c.st);
    DGemmArgs b;
    b.M = N;
    b.N = L;
    b.K = p;
    if (transpose) {
        b.A = static_cast<const double*>(cv.R.p);  // R^T: (n, a) -> R[a + n p]
        b.a_ms = p;
        b.a_ks = 1;
    } else {
        b.A = static_cast<const double*>(cv.C.p);  // C: (n, a) -> C[n + a N]
        b.a_ms = 1;
        b.a_ks = N;
    }
    b.B = t;
    b.b_ks = 1;
    b.b_ns = p;
    b.C = X;
    b.c_ms = 1;
    b.c_ns = ld;
    b.alpha = -1.0;
    b.beta = 1.0;
    launch_dgemm(b, c.st);
    ck(cudaGetLastError(), "projection");
}

// Dense T matrix (rows x cols, column-major) to a device FP64 buffer with
// leading dimension ld (padding rows zero).
template <typename T>
double* upload_dense(Context& c, DevBuf& buf, const T* h, int64_t rows, int64_t cols, int64_t ld) {
    std::vector<double> tmp((size_t)(ld * cols), 0.0);
    for (int64_t q = 0; q < cols; ++q)
        for (int64_t i = 0; i < rows; ++i) tmp[(size_t)(q * ld + i)] = (double)h[q * rows + i];
    double* d = buf.as<double>(std::max<size_t>(tmp.size(), 1));
    h2d(d, tmp.data(), tmp.size(), c.st);
    return d;
}

template <typename T>
void download_dense(Context& c, T* h, const double* d, int64_t rows, int64_t cols, int64_t ld) {
    std::vector<double> tmp((size_t)(ld * cols));
    d2h(tmp.data(), d, tmp.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "download");
    for (int64_t q = 0; q < cols; ++q)
        for (int64_t i = 0; i < rows; ++i) h[q * rows + i] = (T)tmp[(size_t)(q * ld + i)];
}

// inv_j = 1/sqrt(max(eps, ss_j / df)) from ||x_j||^2 and (with covariates)
// proj = R x_j: ss_j + q - 2h (compute_inv_resvar_from_geno_block,
// gwldcore.cpp:3220-3333).
template <typename T>
void inv_from_sumsq(const double* ss, const double* proj, int64_t L, int64_t p, const T* gram,
                    double df, double eps, T* inv_out) {
    for (int64_t j = 0; j < L; ++j) {
        double s2 = ss[j];
        if (proj && p > 0) {
            const double* t = proj + j * p;
            double h = 0.0;
            for (int64_t k = 0; k < p; ++k) h += t[k] * t[k];
            double q = h;
            if (gram) {
                q = 0.0;
                for (int64_t a = 0; a < p; ++a) {
                    double gy = 0.0;
                    for (int64_t b = 0; b < p; ++b) gy += (double)gram[a * p + b] * t[b];
                    q += t[a] * gy;
                }
            }
            s2 += q - 2.0 * h;
        }
        const double var = s2 / df;
        const double safe = std::isnan(var) ? var : (var > eps ? var : eps);
        inv_out[j] = (T)(1.0 / std::sqrt(safe));
    }
}

template <typename T>
void phase1_geno_impl(const T* geno, int64_t N, int64_t L, int blk_start, const T* annot,
                      int64_t annot_rows, int64_t K, const T* inv_right, int v_start, int v_count,
                      int rand_dist, int has_seed, uint64_t seed, T* Xz, int64_t xz_rows,
                      int64_t xz_cols, uint8_t* bin_init, T* inv_out, double eps, const T* Cm,
                      const T* Rm, int64_t p, const T* gram) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (N <= 0 || L < 0) fail(LDS_ERR_ARG, "Invalid external genotype block dimensions in phase1");
    if (L == 0) return;
    if (annot_rows != L) fail(LDS_ERR_ARG, "L mismatch");
    DevBuf dx, dtmp, dp;
    double* X = upload_dense<T>(c, dx, geno, N, L, N);
    std::vector<T> inv((size_t)L);
    if (inv_out) {
        if ((Cm != nullptr) != (Rm != nullptr))
            fail(LDS_ERR_ARG, "C and R must be provided together for fused residual variances");
        if (N <= 1) fail(LDS_ERR_ARG, "Invalid block dimensions in compute_inv_resvar_from_geno_block");
        const bool cov = Cm && Rm && p > 0;
        if (cov && N - p <= 1) fail(LDS_ERR_ARG, "N_eff must be > 1 in fused residual variances");
        const double df = cov ? (double)(N - p - 1) : (double)(N - 1);
        std::vector<double> ss((size_t)L), proj;
        double* dss = dtmp.as<double>((size_t)L);
        launch_col_sumsq(X, N, N, L, dss, c.st);
        d2h(ss.data(), dss, ss.size(), c.st);
        if (cov) {
            DevCov cv;
            upload_cov<T>(c, cv, Cm, Rm, N, p);
            double* pr = dp.as<double>((size_t)(p * L));
            DGemmArgs a;
            a.M = p;
            a.N = L;
            a.K = N;
            a.A = static_cast<const double*>(cv.R.p);
            a.a_ms = 1;
            a.a_ks = p;
            a.B = X;
            a.b_ks = 1;
            a.b_ns = N;
            a.C = pr;
            a.c_ms = 1;
            a.c_ns = p;
            launch_dgemm(a, c.st);
            proj.resize((size_t)(p * L));
            d2h(proj.data(), pr, proj.size(), c.st);
        }
        ck(cudaStreamSynchronize(c.st), "resvar");
        inv_from_sumsq<T>(ss.data(), cov ? proj.data() : nullptr, L, p, gram, df, eps, inv.data());
        std::memcpy(inv_out, inv.data(), sizeof(T) * (size_t)L);
    } else {
        if (!inv_right) fail(LDS_ERR_ARG, "inv_right shape mismatch in phase1");
        std::memcpy(inv.data(), inv_right, sizeof(T) * (size_t)L);
    }
    if (xz_rows != N || xz_cols != K * v_count)
        fail(LDS_ERR_ARG, "Xz2d_chunk shape must be (N, B*v_count)");
    if (v_count <= 0) return;
    const int V = v_count;
    const uint64_t root = has_seed ? seed : std::random_device{}();
    std::vector<double> Z((size_t)(L * V));
    make_probes<T>(root, blk_start, v_start, (int)L, V, rand_dist, Z.data(), L);
    const Csr cs = build_csr<T>(annot, inv.data(), L, K, 0, 1, 1, 1);
    DevBuf dxz, db, di;
    double* Y = upload_dense<T>(c, dxz, Xz, N, K * V, N);
    std::vector<char> touched((size_t)K, 0);
    for (int64_t k = 0; k < K; ++k) {
        const int64_t n = cs.nnz[(size_t)k];
        if (n == 0) continue;
        const int64_t o = cs.bin_off[(size_t)k];
        std::vector<double> Bk((size_t)(n * V));
        for (int64_t cc = 0; cc < V; ++cc)
            for (int64_t r = 0; r < n; ++r)
                Bk[(size_t)(cc * n + r)] =
                    (double)(T)(Z[(size_t)(cc * L + cs.rowind[(size_t)(o + r)])] * cs.sc[(size_t)(o + r)]);
        double* dB = db.as<double>(Bk.size());
        h2d(dB, Bk.data(), Bk.size(), c.st);
        int32_t* dI = di.as<int32_t>((size_t)n);
        h2d(dI, cs.rowind.data() + o, (size_t)n, c.st);
        bool beta1 = true;
        if (bin_init) {
            beta1 = bin_init[k] != 0;
            bin_init[k] = 1;
        }
        DGemmArgs a;
        a.M = N;
        a.N = V;
        a.K = n;
        a.A = X;
        a.a_ms = 1;
        a.a_ks = N;
        a.a_kidx = dI;
        a.B = dB;
        a.b_ks = 1;
        a.b_ns = n;
        a.C = Y + k * V * N;
        a.c_ms = 1;
        a.c_ns = N;
        a.beta = beta1 ? 1.0 : 0.0;
        launch_dgemm(a, c.st);
        ck(cudaStreamSynchronize(c.st), "phase1 dense");  // Bk and the index are reused
        touched[(size_t)k] = 1;
    }
    ck(cudaGetLastError(), "phase1 dense");
    std::vector<double> out((size_t)(N * K * V));
    d2h(out.data(), Y, out.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "phase1 dense");
    for (int64_t k = 0; k < K; ++k) {
        if (!touched[(size_t)k]) continue;
        for (int64_t q = k * V; q < (k + 1) * V; ++q)
            for (int64_t i = 0; i < N; ++i) Xz[q * N + i] = (T)out[(size_t)(q * N + i)];
    }
}

// Left scales, device accumulators and the guarded reduction of a product
// panel W (L x Q on the device), merged into the caller's outputs like
// phase2_bed_impl.
template <typename T>
void dense_p2_finish(Context& c, const double* W, int64_t L, int64_t K, int V, const T* inv_left,
                     int N_denom, T* meansq, int blk_start, double* mc_agg, double* mc_snp,
                     const char* label) {
    double denom = (double)N_denom - 1.0;
    if (denom <= 0.0) denom = 1.0;
    const double inv_denom2 = 1.0 / (denom * denom);
    std::vector<double> ls((size_t)L);
    for (int64_t i = 0; i < L; ++i) {
        const double v = (double)inv_left[i];
        ls[(size_t)i] = (std::isfinite(v) && v > 0.0) ? v * v * inv_denom2 : 0.0;
    }
    DevBuf dls, dacc, dmc;
    double* d_ls = dls.as<double>((size_t)L);
    h2d(d_ls, ls.data(), ls.size(), c.st);
    double* d_acc = dacc.as<double>((size_t)(L * K));
    ck(cudaMemsetAsync(d_acc, 0, sizeof(double) * (size_t)(L * K), c.st), "memset");
    double* d_mc = nullptr;
    if (mc_agg || mc_snp) {
        d_mc = dmc.as<double>((size_t)(L * K));
        ck(cudaMemsetAsync(d_mc, 0, sizeof(double) * (size_t)(L * K), c.st), "memset");
    }
    unsigned long long* g = c.guards.as<unsigned long long>(4);
    ck(cudaMemsetAsync(g, 0, 32, c.st), "memset");
    launch_dense_p2_epilogue(W, L, (int)K, V, d_ls, d_acc, d_mc, g, extreme_warn_env(),
                             drop_extreme_env(), c.st);
    ck(cudaGetLastError(), "launch");
    std::vector<double> upd((size_t)(L * K)), mcv;
    d2h(upd.data(), d_acc, upd.size(), c.st);
    if (d_mc) {
        mcv.resize((size_t)(L * K));
        d2h(mcv.data(), d_mc, mcv.size(), c.st);
    }
    ck(cudaStreamSynchronize(c.st), "phase2 dense");
    report_guards(c, label, blk_start, (int)(blk_start + L));
    for (int64_t i = 0; i < L; ++i)
        for (int64_t k = 0; k < K; ++k)
            meansq[(blk_start + i) * K + k] += (T)upd[(size_t)(i * K + k)];
    if (d_mc) {
        for (int64_t k = 0; k < K; ++k) {
            double agg = 0.0;
            for (int64_t i = 0; i < L; ++i) {
                const double sv = mcv[(size_t)(i * K + k)];
                agg += sv;
                if (mc_snp) mc_snp[(blk_start + i) * K + k] += sv;
            }
            if (mc_agg) mc_agg[k] += agg;
        }
    }
}

template <typename T>
void phase2_geno_impl(T* geno, int64_t N, int64_t L, int blk_start, const T* inv_left,
                      int64_t L_in, int tile_nvecs, const T* Xz, int64_t xz_rows, int64_t xz_cols,
                      T* meansq, int64_t M_rows, int64_t K_in, const T* Cm, const T* Rm, int64_t p,
                      int N_denom, double* mc_agg, double* mc_snp) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (N <= 0 || L < 0) fail(LDS_ERR_ARG, "Invalid external genotype block dimensions in phase2");
    if (L == 0) return;
    DevBuf dx, dtmp, dxz, dw;
    double* X = upload_dense<T>(c, dx, geno, N, L, N);
    if (Cm && Rm && p > 0) {
        // the reference projects the caller's genotype block in place
        DevCov cv;
        upload_cov<T>(c, cv, Cm, Rm, N, p);
        project_cols(c, X, N, L, cv, false, dtmp);
        download_dense<T>(c, geno, X, N, L, N);
    }
    if (L_in != L) fail(LDS_ERR_ARG, "inv_left shape mismatch in phase2_accum_XtXz_bed");
    if (xz_rows != N) fail(LDS_ERR_ARG, "Xz2d shape mismatch in phase2_accum_XtXz_bed");
    const int64_t Q = xz_cols;
    if (tile_nvecs <= 0 || Q % tile_nvecs)
        fail(LDS_ERR_ARG, "Xz2d col count must be a multiple of tile_nvecs");
    const int64_t K = Q / tile_nvecs;
    if (K_in != K) fail(LDS_ERR_ARG, "meansq_accum shape mismatch in phase2_accum_XtXz_bed");
    if (blk_start + L > M_rows) fail(LDS_ERR_ARG, "meansq_accum rows smaller than SNP count");
    if (K > 512) fail(LDS_ERR_ARG, "B too large for fixed seg buffers in phase2_accum_XtXz_bed");
    double* Y = upload_dense<T>(c, dxz, Xz, N, Q, N);
    double* W = dw.as<double>((size_t)(L * Q));
    DGemmArgs a;
    a.M = L;
    a.N = Q;
    a.K = N;
    a.A = X;  // X^T: (j, n) -> X[n + j N]
    a.a_ms = N;
    a.a_ks = 1;
    a.B = Y;
    a.b_ks = 1;
    a.b_ns = N;
    a.C = W;
    a.c_ms = 1;
    a.c_ns = L;
    launch_dgemm(a, c.st);
    dense_p2_finish<T>(c, W, L, K, tile_nvecs, inv_left, N_denom, meansq, blk_start, mc_agg,
                       mc_snp, "accum");
}

// GRM panel products (apply_grm_bed_panel_impl, gwldcore.cpp:1134-1254, and
// its Mailman form :1256-1497): out = P X D X^T P V with D = diag(inv_j^2 / M)
// over SNPs [0, nsnps) and P = I - C R when covariates are given.  X^T V runs
// on the phase-2 tensor-core kernel's exact raw-product mode and X (D coef) on
// the phase-1 kernel.
template <typename T>
void apply_grm_impl(const char* bed_prefix, const char* fam_path, int nsnps, int step_size,
                    const int64_t* row_sel, int64_t n_row_sel, int ddof, const T* inv_all,
                    int64_t n_inv, const T* panel_in, T* panel_out, int64_t rows, int64_t Q,
                    const T* Cm, const T* Rm, int64_t p, int impute, int has_iseed, uint64_t iseed,
                    const char* name) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    int64_t M = 0;
    Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel, impute,
                                    has_iseed ? iseed : 0ULL, ddof, &M);
    if (nsnps < 0 || nsnps > M) fail(LDS_ERR_ARG, "nsnps is out of range in %s", name);
    if (step_size <= 0) fail(LDS_ERR_ARG, "step_size must be > 0 in %s", name);
    const int64_t N = P.g.N, Np = P.g.N_pad;
    if (N <= 0) fail(LDS_ERR_ARG, "No rows selected in %s", name);
    if (n_inv < nsnps) fail(LDS_ERR_ARG, "inv_all shape mismatch in %s", name);
    if (rows != N) fail(LDS_ERR_ARG, "panel row mismatch in %s", name);
    for (int64_t i = 0; i < N * Q; ++i) panel_out[i] = T(0);
    if (Q == 0 || nsnps == 0) return;
    DevCov cv;
    upload_cov<T>(c, cv, Cm, Rm, N, p);
    DevBuf dv, dtmp;
    double* V = upload_dense<T>(c, dv, panel_in, N, Q, Np);
    project_cols(c, V, Np, Q, cv, false, dtmp);
    std::vector<double> Vh((size_t)(N * Q));
    for (int64_t q = 0; q < Q; ++q)
        d2h(Vh.data() + q * N, V + q * Np, (size_t)N, c.st);
    ck(cudaStreamSynchronize(c.st), "grm panel");
    const std::vector<double> coef = snp_products(c, P, 0, nsnps, Vh, Q);  // nsnps x Q row-major
    const double invM = 1.0 / (double)nsnps;
    std::vector<T> w((size_t)nsnps), ones((size_t)nsnps, T(1));
    for (int64_t j = 0; j < nsnps; ++j) {
        const double ij = (double)inv_all[j];
        double x = ij * ij * invM;
        if (!std::isfinite(x) || x <= 0.0) x = 0.0;
        w[(size_t)j] = (T)x;
    }
    std::vector<double> Z((size_t)(nsnps * Q));
    for (int64_t j = 0; j < nsnps; ++j)
        for (int64_t q = 0; q < Q; ++q) Z[(size_t)(q * nsnps + j)] = (double)(T)coef[(size_t)(j * Q + q)];
    const int Vp = (int)round_up(Q, kColTile);
    const Csr cs = build_csr<T>(ones.data(), w.data(), nsnps, 1, 0, Vp, c.slices, kSnpStep,
                                P.constant.data());
    if (cs.nnz[0] == 0) return;
    run_phase1(c, P, cs, 1, (int)Q, Z.data(), nsnps, nsnps, 0);
    double* Y = static_cast<double*>(c.y.p);
    project_cols(c, Y, Np, Q, cv, false, dtmp);
    std::vector<double> out((size_t)(Np * Q));
    d2h(out.data(), Y, out.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "grm panel");
    for (int64_t q = 0; q < Q; ++q)
        for (int64_t i = 0; i < N; ++i) panel_out[q * N + i] = (T)out[(size_t)(q * Np + i)];
}

// mu22 (precompute_residual_variances_bed_impl, gwldcore.cpp:3421-3563):
// S = sum_j (x_j o x_j) a_jk inv_j^2 over the (projected) standardized
// genotypes, mu22[a][b] = (S^T S)[a][b] / (N Msum_a Msum_b).
template <typename T>
void mu22_impl(Context& c, const Prepared& P, int64_t nsnps, const T* inv, const T* annot,
               int64_t B, const T* Cm, const T* Rm, int64_t p, double* mu22) {
    const int64_t N = P.g.N;
    std::vector<double> Msum((size_t)B, 0.0);
    for (int64_t j = 0; j < nsnps; ++j)
        for (int64_t k = 0; k < B; ++k) Msum[(size_t)k] += (double)annot[j * B + k];
    DevCov cv;
    upload_cov<T>(c, cv, Cm, Rm, N, p);
    const int64_t Lb = std::max<int64_t>(1, std::min<int64_t>(std::max<int64_t>(nsnps, 1),
                                                              (int64_t)(256u << 20) / (8 * N)));
    DevBuf dx, dtmp, dwt, ds, dss;
    double* X = dx.as<double>((size_t)(N * Lb));
    double* S = ds.as<double>((size_t)(N * B));
    ck(cudaMemsetAsync(S, 0, sizeof(double) * (size_t)(N * B), c.st), "memset");
    double* Wd = dwt.as<double>((size_t)(Lb * B));
    std::vector<double> Wh((size_t)(Lb * B));
    for (int64_t j0 = 0; j0 < nsnps; j0 += Lb) {
        const int64_t L = std::min(Lb, nsnps - j0);
        launch_decode_standardized(P.g, j0, L, static_cast<const double*>(P.d_mean.p),
                                   static_cast<const double*>(P.d_sdinv.p), X, N, c.st);
        project_cols(c, X, N, L, cv, false, dtmp);
        for (int64_t k = 0; k < B; ++k)
            for (int64_t j = 0; j < L; ++j) {
                const double iv = (double)inv[j0 + j];
                Wh[(size_t)(k * L + j)] = (double)annot[(j0 + j) * B + k] * (iv * iv);
            }
        ck(cudaStreamSynchronize(c.st), "mu22");  // Wd is rewritten
        h2d(Wd, Wh.data(), (size_t)(L * B), c.st);
        DGemmArgs a;
        a.M = N;
        a.N = B;
        a.K = L;
        a.A = X;
        a.a_ms = 1;
        a.a_ks = N;
        a.a_square = 1;
        a.B = Wd;
        a.b_ks = 1;
        a.b_ns = L;
        a.C = S;
        a.c_ms = 1;
        a.c_ns = N;
        a.beta = 1.0;
        launch_dgemm(a, c.st);
    }
    double* SS = dss.as<double>((size_t)(B * B));
    DGemmArgs g;
    g.M = B;
    g.N = B;
    g.K = N;
    g.A = S;
    g.a_ms = N;
    g.a_ks = 1;
    g.B = S;
    g.b_ks = 1;
    g.b_ns = N;
    g.C = SS;
    g.c_ms = 1;
    g.c_ns = B;
    launch_dgemm(g, c.st);
    ck(cudaGetLastError(), "mu22");
    std::vector<double> h((size_t)(B * B));
    d2h(h.data(), SS, h.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "mu22");
    for (int64_t a = 0; a < B; ++a)
        for (int64_t b = 0; b < B; ++b) {
            const double den = (double)N * Msum[(size_t)a] * Msum[(size_t)b];
            double v = 0.0;
            if (den != 0.0) {
                v = h[(size_t)(a + b * B)] / den;
                if (!std::isfinite(v)) v = 0.0;
            }
            mu22[a * B + b] = v;
        }
}

template <typename Tann>
void block_corrections_impl(const double* meansq, const double* mu22, const Tann* annot,
                            int64_t M, int64_t B, int N, double d, double* R2, double* rho2,
                            double* bias, double* delta) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (N <= 1) fail(LDS_ERR_ARG, "N must be > 1 in compute_block_corrections_binary");
    if (B <= 0) return;
    DevBuf dm, du, da, dout;
    double* m = dm.as<double>((size_t)std::max<int64_t>(M * B, 1));
    h2d(m, meansq, (size_t)(M * B), c.st);
    double* u = du.as<double>((size_t)(B * B));
    h2d(u, mu22, (size_t)(B * B), c.st);
    Tann* an = da.as<Tann>((size_t)std::max<int64_t>(M * B, 1));
    h2d(an, annot, (size_t)(M * B), c.st);
    double* o = dout.as<double>((size_t)(4 * B * B));
    launch_block_corrections<Tann>(m, u, an, M, (int)B, (double)N, d, o, o + B * B, o + 2 * B * B,
                                   o + 3 * B * B, c.st);
    ck(cudaGetLastError(), "launch");
    d2h(R2, o, (size_t)(B * B), c.st);
    d2h(rho2, o + B * B, (size_t)(B * B), c.st);
    d2h(bias, o + 2 * B * B, (size_t)(B * B), c.st);
    d2h(delta, o + 3 * B * B, (size_t)(B * B), c.st);
    ck(cudaStreamSynchronize(c.st), "block corrections");
}

template <typename T>
void phase1_bed_impl(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
                     const int64_t* row_sel, int64_t n_row_sel, int ddof, const T* annot,
                     int64_t annot_rows, int64_t K, const T* inv_right, int v_start, int v_count,
                     int rand_dist, int has_seed, uint64_t seed, T* Xz, int64_t xz_rows,
                     int64_t xz_cols, uint8_t* bin_init, int impute, int has_iseed,
                     uint64_t iseed, T* inv_out, double resvar_eps, const T* Cm = nullptr,
                     const T* Rm = nullptr, int64_t p = 0, const T* gram = nullptr,
                     int project_right = 0) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (impute != LDS_IMPUTE_MEAN && impute != LDS_IMPUTE_HWE)
        fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
    int64_t M = 0;
    Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel, impute,
                                    has_iseed ? iseed : 0ULL, ddof, &M);
    if (blk_end > M) fail(LDS_ERR_ARG, "blk_end exceeds #SNPs in BIM");
    if (blk_end <= blk_start) return;
    const int64_t L = blk_end - blk_start;
    // project_right (gwldcore.cpp:1633-1650): the block's genotypes are
    // projected, X <- (I - C R) X, before the products; by linearity the
    // block's contribution to the sketch is projected instead.
    const bool proj = project_right && Cm && Rm && p > 0;
    if (proj && inv_out)
        fail(LDS_ERR_ARG, "Fused residual variance is incompatible with project_right=True");
    if (annot_rows != L) fail(LDS_ERR_ARG, "L mismatch");
    std::vector<T> inv((size_t)L);
    if (inv_out) {
        if (Cm && Rm && p > 0)
            inv_resvar_fused_cov<T>(c, P, blk_start, L, Cm, Rm, p, gram, resvar_eps, inv.data());
        else
            for (int64_t i = 0; i < L; ++i) inv[(size_t)i] = inv_resvar<T>(P, blk_start + i, resvar_eps);
        std::memcpy(inv_out, inv.data(), sizeof(T) * (size_t)L);
    } else {
        if (!inv_right) fail(LDS_ERR_ARG, "inv_right shape mismatch in phase1");
        std::memcpy(inv.data(), inv_right, sizeof(T) * (size_t)L);
    }
    if (xz_rows != P.g.N || xz_cols != K * v_count)
        fail(LDS_ERR_ARG, "Xz2d_chunk shape must be (N, B*v_count)");
    if (v_count <= 0) return;
    const int S = c.slices;
    const int Vp = (int)round_up(v_count, kColTile);
    Csr csr = build_csr<T>(annot, inv.data(), L, K, blk_start, Vp, S, kSnpStep, P.constant.data());
    const uint64_t root = has_seed ? seed : std::random_device{}();
    std::vector<double> Z((size_t)(L * v_count));
    make_probes<T>(root, blk_start, v_start, (int)L, v_count, rand_dist, Z.data(), L);
    run_phase1(c, P, csr, K, v_count, Z.data(), L, L, blk_start);
    const int64_t N = P.g.N;
    if (proj) {
        DevCov cv;
        upload_cov<T>(c, cv, Cm, Rm, N, p);
        DevBuf tmp;
        project_cols(c, static_cast<double*>(c.y.p), P.g.N_pad, K * v_count, cv, false, tmp);
    }
    // Download the block's contribution and merge with beta semantics.
    std::vector<double> D((size_t)(N * K * v_count));
    const double* Y = static_cast<double*>(c.y.p);
    for (int64_t q = 0; q < K * v_count; ++q)
        d2h(D.data() + q * N, Y + q * P.g.N_pad, (size_t)N, c.st);
    ck(cudaStreamSynchronize(c.st), "phase1");
    for (int64_t k = 0; k < K; ++k) {
        if (csr.nnz[(size_t)k] == 0) continue;
        bool beta1 = true;
        if (bin_init) {
            beta1 = bin_init[k] != 0;
            bin_init[k] = 1;
        }
        for (int64_t cc = 0; cc < v_count; ++cc) {
            T* dst = Xz + (k * v_count + cc) * N;
            const double* src = D.data() + (k * v_count + cc) * N;
            if (beta1)
                for (int64_t n = 0; n < N; ++n) dst[n] = (T)((double)dst[n] + src[n]);
            else
                for (int64_t n = 0; n < N; ++n) dst[n] = (T)src[n];
        }
    }
}

template <typename T>
void phase2_bed_impl(const char* bed_prefix, const char* fam_path, int blk_start, int blk_end,
                     const int64_t* row_sel, int64_t n_row_sel, int ddof, const T* inv_left,
                     int64_t L_in, int tile_nvecs, const T* Xz, int64_t xz_rows, int64_t xz_cols,
                     T* meansq, int64_t M_rows, int64_t K_in, int N_denom, int impute,
                     int has_iseed, uint64_t iseed, double* mc_agg, double* mc_snp,
                     const T* Cm = nullptr, const T* Rm = nullptr, int64_t p = 0,
                     int proj_sketch = 0, double post_scale = 1.0, const char* label = "accum") {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (impute != LDS_IMPUTE_MEAN && impute != LDS_IMPUTE_HWE)
        fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
    int64_t M = 0;
    Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel, impute,
                                    has_iseed ? iseed : 0ULL, ddof, &M);
    if (blk_end > M) fail(LDS_ERR_ARG, "blk_end exceeds #SNPs in BIM");
    if (blk_end <= blk_start) return;
    const int64_t L = blk_end - blk_start;
    if (L_in != L) fail(LDS_ERR_ARG, "inv_left shape mismatch in phase2_accum_XtXz_bed");
    if (xz_rows != P.g.N) fail(LDS_ERR_ARG, "Xz2d shape mismatch in phase2_accum_XtXz_bed");
    const int64_t Q = xz_cols;
    if (tile_nvecs <= 0 || Q % tile_nvecs)
        fail(LDS_ERR_ARG, "Xz2d col count must be a multiple of tile_nvecs");
    const int64_t K = Q / tile_nvecs;
    if (K_in != K) fail(LDS_ERR_ARG, "meansq_accum shape mismatch in phase2_accum_XtXz_bed");
    if (blk_end > M_rows) fail(LDS_ERR_ARG, "meansq_accum rows smaller than SNP count");
    if (K > 512) fail(LDS_ERR_ARG, "B too large for fixed seg buffers in phase2_accum_XtXz_bed");
    const int64_t N = P.g.N, Np = P.g.N_pad;
    // Sketch to device (FP64, padded rows zero).
    std::vector<double> y((size_t)(Np * Q), 0.0);
    for (int64_t q = 0; q < Q; ++q)
        for (int64_t n = 0; n < N; ++n) y[(size_t)(q * Np + n)] = (double)Xz[q * N + n];
    double* dY = c.y.as<double>((size_t)(Np * Q));
    h2d(dY, y.data(), y.size(), c.st);
    if (Cm && Rm && p > 0) {
        // Work = ((I - C R) X)^T Xz = X^T (I - C R)^T Xz for the dense form
        // (gwldcore.cpp:2376-2390); the Mailman form projects the sketch,
        // Xz <- (I - C R) Xz (:615-638).
        DevCov cv;
        upload_cov<T>(c, cv, Cm, Rm, N, p);
        DevBuf tmp;
        project_cols(c, dY, Np, Q, cv, proj_sketch == 0, tmp);
    }
    quantize_sketch(c, P, K, tile_nvecs);
    // Left scales.
    double denom = (double)N_denom - 1.0;
    if (denom <= 0.0) denom = 1.0;
    const double inv_denom2 = 1.0 / (denom * denom);
    std::vector<double> ls((size_t)M, 0.0);
    for (int64_t i = 0; i < L; ++i) {
        const double v = (double)inv_left[i];
        ls[(size_t)(blk_start + i)] = (std::isfinite(v) && v > 0.0) ? v * v * inv_denom2 : 0.0;
    }
    double* d_ls = c.lscale.as<double>((size_t)M);
    h2d(d_ls, ls.data(), (size_t)M, c.st);
    double* d_acc = c.accum.as<double>((size_t)(L * K));
    ck(cudaMemsetAsync(d_acc, 0, sizeof(double) * (size_t)(L * K), c.st), "memset");
    double* d_mc = nullptr;
    if (mc_agg || mc_snp) {
        d_mc = c.mc.as<double>((size_t)(L * K));
        ck(cudaMemsetAsync(d_mc, 0, sizeof(double) * (size_t)(L * K), c.st), "memset");
    }
    ck(cudaMemsetAsync(c.guards.as<unsigned long long>(4), 0, 32, c.st), "memset");
    run_phase2(c, P, K, tile_nvecs, blk_start, blk_end, blk_start, d_acc, d_mc, d_ls);
    std::vector<double> upd((size_t)(L * K)), mcv;
    d2h(upd.data(), d_acc, upd.size(), c.st);
    if (d_mc) {
        mcv.resize((size_t)(L * K));
        d2h(mcv.data(), d_mc, mcv.size(), c.st);
    }
    ck(cudaStreamSynchronize(c.st), "phase2");
    report_guards(c, label, blk_start, blk_end);
    for (int64_t i = 0; i < L; ++i)
        for (int64_t k = 0; k < K; ++k)
            meansq[(blk_start + i) * K + k] += (T)(upd[(size_t)(i * K + k)] * post_scale);
    if (d_mc) {
        for (int64_t k = 0; k < K; ++k) {
            double agg = 0.0;
            for (int64_t i = 0; i < L; ++i) {
                const double s = mcv[(size_t)(i * K + k)];
                agg += s;
                if (mc_snp) mc_snp[(blk_start + i) * K + k] += s;
            }
            if (mc_agg) mc_agg[k] += agg;
        }
    }
}

template <typename T>
void resvar_impl(const char* bed_prefix, const char* fam_path, int nsnps, const int64_t* row_sel,
                 int64_t n_row_sel, int ddof, double eps, int impute, int has_iseed,
                 uint64_t iseed, T* inv_out, const T* Cm = nullptr, const T* Rm = nullptr,
                 int64_t p = 0, double* snp_var = nullptr, const T* annot_all = nullptr,
                 int64_t annot_rows = 0, int64_t B = 0, double* mu22 = nullptr) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    int64_t M = 0;
    Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel, impute,
                                    has_iseed ? iseed : 0ULL, ddof, &M);
    if (nsnps > M) fail(LDS_ERR_ARG, "nsnps exceeds #SNPs in BIM");
    if (P.g.N <= 1) fail(LDS_ERR_ARG, "Invalid block dimensions in compute_inv_resvar_from_geno_block");
    if ((Cm != nullptr) != (Rm != nullptr)) fail(LDS_ERR_ARG, "C and R must be provided together");
    if (mu22) {
        if (!annot_all) fail(LDS_ERR_ARG, "annot_all must be provided when compute_mu22=True");
        if (annot_rows != nsnps)
            fail(LDS_ERR_ARG, "annot_all shape mismatch in precompute_residual_variances_bed");
        if (B <= 0) fail(LDS_ERR_ARG, "annot_all must have at least one column");
    }
    if (Cm && Rm && p > 0) {
        inv_resvar_projected_cov<T>(c, P, nsnps, Cm, Rm, p, eps, inv_out, snp_var);
    } else {
        for (int64_t j = 0; j < nsnps; ++j) {
            inv_out[j] = inv_resvar<T>(P, j, eps);
            if (snp_var) snp_var[j] = sumsq_std<T>(P, j) > 0.0 ? 1.0 : 0.0;
        }
    }
    if (mu22) mu22_impl<T>(c, P, nsnps, inv_out, annot_all, B, Cm, Rm, p, mu22);
}

// ---------------------------------------------------------------------------
// Genome-wide estimator as geno handle + plan + execute.  A plan holds every
// device input of the kernels (CSR lists, probes, left scales), so execute()
// is a pure sequence of asynchronous launches on the library stream — the
// unit the benchmark times and that can be captured in a CUDA graph.
// ---------------------------------------------------------------------------
struct GwPlan {
    std::shared_ptr<Prepared> P;
    int64_t K = 0;
    int nvecs = 0, S = 4, as_float = 0, with_mc = 0;
    std::vector<int> vt;
    std::vector<double> inv, Mk;
    struct Tile {
        int V = 0, Vp = 0;
        Csr csr;
        DevBuf rowind, sc, binoff, wqoff, z, wq, wcs;
        int64_t lmax = 0;     // tcgen05 phase 1: padded member-list length
        CUtensorMap tmW;      // tcgen05 phase 1: weight digits
    };
    std::vector<std::unique_ptr<Tile>> tiles;
    DevBuf y, yq, ycs, accum, mc, lscale, guards, status;
    DevBuf colsum;                   // sketch digit column sums (images with complete tiles)
    bool umma = false;
    CUtensorMap tmA;
    // One set of events per execute (up to kMaxTimed executes between reads):
    // a start event and one after each kernel of each V-tile.
    static constexpr int kMaxTimed = 64;
    std::vector<std::vector<cudaEvent_t>> evsets;
    int pending = 0;
    double kernel_ms[4] = {0, 0, 0, 0};  // weights, phase 1, sketch digits, phase 2
    // Product checksums (lds_gw_plan_set_checks), as for windowed plans: lhs
    // from the phase-2 epilogue, rhs from the CUDA-core pass; the rows form
    // one window (a tile table of 128-SNP tiles).  chk_evsets[p][t] closes
    // V-tile t's phase 2 before its check kernels.
    int check = 0, executed = 0;
    // Phase-2 CTA order per bins-per-CTA value (as for windowed batches: chunks
    // of 4 bin groups, all row tiles, the chunk's bin groups).
    std::vector<int> work_nb;
    std::vector<std::unique_ptr<DevBuf>> work;
    std::vector<int64_t> n_work;
    DevBuf chk_lhs, chk_rhs, chk_u, chk_tiles;
    int64_t chk_ntiles = 0;
    std::vector<std::vector<cudaEvent_t>> chk_evsets;
    double check_ms = 0.0;
    int64_t snp_offset = 0;  // index of SNP 0 of this image in the whole fileset (SNP shards)
    ~GwPlan() {
        for (auto& s : evsets)
            for (cudaEvent_t e : s) cudaEventDestroy(e);
        for (auto& s : chk_evsets)
            for (cudaEvent_t e : s) cudaEventDestroy(e);
    }
};

std::map<int64_t, std::shared_ptr<Prepared>>& geno_table() {
    static std::map<int64_t, std::shared_ptr<Prepared>> t;
    return t;
}
std::map<int64_t, std::unique_ptr<GwPlan>>& plan_table() {
    static std::map<int64_t, std::unique_ptr<GwPlan>> t;
    return t;
}
int64_t next_handle() {
    static int64_t h = 0;
    return ++h;
}

std::unique_ptr<GwPlan> plan_create(Context& c, std::shared_ptr<Prepared> P, const double* annot,
                                    int64_t K, int nvecs, int step, int vtile, uint64_t seed,
                                    int dist, double eps, int as_float, int with_mc,
                                    int64_t snp_offset = 0) {
    const int64_t M = P->g.M, N = P->g.N;
    if (nvecs <= 0 || step <= 0 || K <= 0 || M <= 0) fail(LDS_ERR_ARG, "invalid sizes");
    if (snp_offset < 0 || snp_offset % step != 0)
        fail(LDS_ERR_ARG, "a SNP shard must start on a block boundary (a multiple of step_size)");
    if (K > 512) fail(LDS_ERR_ARG, "B too large for fixed seg buffers in phase2_accum_XtXz_bed");
    auto pl = std::make_unique<GwPlan>();
    pl->P = P;
    pl->K = K;
    pl->nvecs = nvecs;
    pl->S = c.slices;
    pl->as_float = as_float;
    pl->with_mc = with_mc;
    pl->snp_offset = snp_offset;
    {
        int width = std::min(nvecs, vtile > 0 ? vtile : nvecs);
        if (width >= 64) width = std::max(64, (width / 64) * 64);
        for (int s = 0; s < nvecs; s += width) pl->vt.push_back(std::min(width, nvecs - s));
    }
    // Residual variances (the reference fuses them into the first phase-1
    // pass; same values), rounded to the working type.
    pl->inv.resize((size_t)M);
    for (int64_t j = 0; j < M; ++j)
        pl->inv[(size_t)j] =
            as_float ? (double)inv_resvar<float>(*P, j, eps) : inv_resvar<double>(*P, j, eps);
    pl->Mk.assign((size_t)K, 0.0);
    for (int64_t j = 0; j < M; ++j)
        for (int64_t k = 0; k < K; ++k) pl->Mk[(size_t)k] += annot[j * K + k];
    // Left scales (gwldcore.cpp:2436-2445) with N_denom = N - ddof + 1.
    const double denom = std::max(1.0, (double)(N - P->ddof + 1) - 1.0);
    const double inv_denom2 = 1.0 / (denom * denom);
    std::vector<double> ls((size_t)M);
    for (int64_t j = 0; j < M; ++j) {
        const double v = pl->inv[(size_t)j];
        ls[(size_t)j] = (std::isfinite(v) && v > 0.0) ? v * v * inv_denom2 : 0.0;
    }
    h2d(pl->lscale.as<double>((size_t)M), ls.data(), (size_t)M, c.st);
    std::vector<float> annot_f, inv_f;
    if (as_float) {
        annot_f.assign(annot, annot + M * K);
        inv_f.resize((size_t)M);
        for (int64_t j = 0; j < M; ++j) inv_f[(size_t)j] = (float)pl->inv[(size_t)j];
    }
    const int nblk = (int)((M + step - 1) / step);
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    int vmax = 0, v0 = 0;
    for (int V : pl->vt) {
        vmax = std::max(vmax, V);
        auto t = std::make_unique<GwPlan::Tile>();
        t->V = V;
        t->Vp = (int)round_up(V, kColTile);
        const bool tc = (p2_impl() == 1 && pl->S == 4);
        const int64_t pad = tc ? 128 : kSnpStep;
        const uint8_t* cst = P->constant.data();
        t->csr = as_float
            ? build_csr<float>(annot_f.data(), inv_f.data(), M, K, 0, t->Vp, pl->S, pad, cst)
            : build_csr<double>(annot, pl->inv.data(), M, K, 0, t->Vp, pl->S, pad, cst);
        // Probe streams per SNP block (mt19937_64), keyed by the block's start
        // in the whole fileset (make_seed, gwldcore.cpp:452-458): Rademacher
        // streams on the device, Gaussian ones on host threads.
        std::vector<double> Z;
        if (dist == LDS_DIST_RADEMACHER) {
            std::vector<ProbeUnit> units((size_t)nblk);
            for (int b = 0; b < nblk; ++b) {
                const int s = b * step;
                units[(size_t)b] = {s, (int32_t)std::min<int64_t>(step, M - s), 0,
                                    probe_seed(seed, (int)(snp_offset + s), v0)};
            }
            device_rademacher(c, units, V, t->z.as<double>((size_t)(M * V)), M);
        } else {
            Z.resize((size_t)(M * V));
            std::vector<std::thread> th;
            std::atomic<int> next{0};
            for (unsigned w = 0; w < hw; ++w)
                th.emplace_back([&] {
                    for (int b; (b = next.fetch_add(1)) < nblk;) {
                        const int s = b * step;
                        const int L = (int)std::min<int64_t>(step, M - s);
                        std::vector<double> blk((size_t)L * V);
                        const int gs = (int)(snp_offset + s);
                        if (as_float) make_probes<float>(seed, gs, v0, L, V, dist, blk.data(), L);
                        else make_probes<double>(seed, gs, v0, L, V, dist, blk.data(), L);
                        for (int cc = 0; cc < V; ++cc)
                            std::memcpy(&Z[(size_t)cc * M + s], &blk[(size_t)cc * L],
                                        sizeof(double) * L);
                    }
                });
            for (auto& x : th) x.join();
        }
        const Csr& cs = t->csr;
        const size_t nm = std::max<size_t>(cs.rowind.size(), 1);
        h2d(t->rowind.as<int32_t>(nm), cs.rowind.data(), cs.rowind.size(), c.st);
        h2d(t->sc.as<double>(nm), cs.sc.data(), cs.sc.size(), c.st);
        h2d(t->binoff.as<int64_t>(cs.bin_off.size()), cs.bin_off.data(), cs.bin_off.size(), c.st);
        h2d(t->wqoff.as<int64_t>(cs.wq_off.size()), cs.wq_off.data(), cs.wq_off.size(), c.st);
        if (!Z.empty()) h2d(t->z.as<double>(Z.size()), Z.data(), Z.size(), c.st);
        if (tc) {
            for (int64_t kk = 0; kk < K; ++kk)
                t->lmax = std::max(t->lmax, cs.bin_off[(size_t)kk + 1] - cs.bin_off[(size_t)kk]);
            t->lmax = std::max<int64_t>(t->lmax, 128);
            const int nc = umma::ncolp_for(V);
            const size_t bytes = (size_t)(K * 2 * nc) * (size_t)t->lmax;
            int8_t* wq = t->wq.as<int8_t>(bytes);
            ck(cudaMemsetAsync(wq, 0, bytes, c.st), "memset weights");
            t->wcs.as<double>((size_t)(K * V));
            t->tmW = make_map_2d(wq, (uint64_t)t->lmax, (uint64_t)(K * 2 * nc), (uint64_t)t->lmax,
                                 128, (uint32_t)std::min(256, nc), CU_TENSOR_MAP_SWIZZLE_128B);
        } else {
            t->wq.as<int8_t>((size_t)std::max<int64_t>(cs.wq_bytes, 16));
            t->wcs.as<double>((size_t)(K * t->Vp));
        }
        ck(cudaStreamSynchronize(c.st), "plan upload");  // Z is a stack temporary
        pl->tiles.push_back(std::move(t));
        v0 += V;
    }
    const int vpmax = (int)round_up(vmax, kColTile);
    pl->umma = (p2_impl() == 1 && pl->S == 4);
    pl->y.as<double>((size_t)(P->g.N_pad * K * vmax));
    if (pl->umma) {
        const int ncolp = umma::ncolp_for(vmax);
        int8_t* yq = pl->yq.as<int8_t>((size_t)(K * ncolp * P->g.N_pad));
        pl->ycs.as<double>((size_t)(K * vmax));
        if (P->has_complete) pl->colsum.as<int>((size_t)(K * ncolp));
        pl->tmA = make_map_2d(P->g.codes, (uint64_t)P->g.nbp, (uint64_t)P->g.M_pad,
                              (uint64_t)P->g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
        ck(cudaMemsetAsync(pl->status.as<unsigned>(1), 0, 4, c.st), "memset");
        // phase-2 CTA orders, one per bins-per-CTA value of the V-tiles
        for (const auto& t : pl->tiles) {
            const int nb = umma::p2_bins_per_cta_grouped(umma::ncolp_for(t->V), (int)K);
            if (std::find(pl->work_nb.begin(), pl->work_nb.end(), nb) != pl->work_nb.end()) continue;
            const int64_t tiles = (M + 127) / 128;
            const int groups = (int)((K + nb - 1) / nb);
            // chunks of about 4 bins, so that the sketch columns the running
            // CTAs share stay in L2 (4 bins x 208 columns x 50k samples: 42 MB)
            const int chunk = std::max(1, 4 / nb);
            std::vector<int2> order;
            for (int g0 = 0; g0 < groups; g0 += chunk)
                for (int64_t tl = 0; tl < tiles; ++tl)
                    for (int g = g0; g < std::min(groups, g0 + chunk); ++g)
                        order.push_back(make_int2((int)tl, g));
            auto buf = std::make_unique<DevBuf>();
            h2d(buf->as<int2>(order.size()), order.data(), order.size(), c.st);
            pl->work_nb.push_back(nb);
            pl->work.push_back(std::move(buf));
            pl->n_work.push_back((int64_t)order.size());
        }
    } else {
        pl->yq.as<int8_t>((size_t)(pl->S * K * vpmax * P->g.N_pad));
        pl->ycs.as<double>((size_t)(K * vpmax));
    }
    pl->accum.as<double>((size_t)(M * K));
    if (with_mc) pl->mc.as<double>((size_t)(M * K));
    pl->guards.as<unsigned long long>(2);
    ck(cudaStreamSynchronize(c.st), "plan");
    return pl;
}

// Zero the plan's accumulators before the first V-tile of an estimate.
void plan_zero(Context& c, GwPlan& pl) {
    const int64_t M = pl.P->g.M, K = pl.K;
    ck(cudaMemsetAsync(pl.accum.p, 0, sizeof(double) * (size_t)(M * K), c.st), "memset");
    if (pl.check) {
        ck(cudaMemsetAsync(pl.chk_lhs.p, 0, sizeof(unsigned long long) * 2 * (size_t)M, c.st), "memset");
        ck(cudaMemsetAsync(pl.chk_rhs.p, 0, sizeof(unsigned long long) * 2 * (size_t)M, c.st), "memset");
    }
    if (pl.with_mc) ck(cudaMemsetAsync(pl.mc.p, 0, sizeof(double) * (size_t)(M * K), c.st), "memset");
    ck(cudaMemsetAsync(pl.guards.p, 0, 16, c.st), "memset");
}

// Phase 1 of V-tile ti: the weights, then the sketch y (N_pad x K*V,
// column-major, column k*V + v) over this image's SNPs.  ev (may be NULL)
// receives one event after each kernel.
void plan_enqueue_phase1(Context& c, GwPlan& pl, size_t ti, double* y, cudaEvent_t* ev, int& e) {
    Prepared& P = *pl.P;
    const int64_t M = P.g.M, K = pl.K;
    GwPlan::Tile& t = *pl.tiles[ti];
    P1Weights w;
    w.K = (int)K;
    w.V = t.V;
    w.Vp = t.Vp;
    w.S = pl.S;
    w.rowind = static_cast<int32_t*>(t.rowind.p);
    w.sc = static_cast<double*>(t.sc.p);
    w.bin_off = static_cast<int64_t*>(t.binoff.p);
    w.wq_off = static_cast<int64_t*>(t.wqoff.p);
    w.wq = static_cast<int8_t*>(t.wq.p);
    w.colscale = static_cast<double*>(t.wcs.p);
    if (pl.umma) {
        const int nc = umma::ncolp_for(t.V);
        umma::P1UWeights uw;
        uw.K = (int)K;
        uw.V = t.V;
        uw.ncolp = nc;
        uw.lmax = t.lmax;
        uw.rowind = w.rowind;
        uw.sc = w.sc;
        uw.bin_off = w.bin_off;
        uw.wq = w.wq;
        uw.colscale = w.colscale;
        umma::launch_p1_weights4(uw, static_cast<double*>(P.d_mean.p),
                                 static_cast<double*>(P.d_sdinv.p), static_cast<double*>(t.z.p), M,
                                 c.st);
        if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
        umma::P1UArgs pa;
        pa.K = (int)K;
        pa.V = t.V;
        pa.ncolp = nc;
        pa.ngroups = (nc + 255) / 256;
        pa.box_rows = std::min(256, nc);
        pa.nbp = P.g.nbp;
        pa.N_pad = P.g.N_pad;
        pa.bin_off = w.bin_off;
        pa.rowind = w.rowind;
        pa.codes = P.g.codes;
        pa.colscale = w.colscale;
        pa.Y = y;
        pa.status = static_cast<unsigned*>(pl.status.p);
        pa.m_pad = P.g.M_pad;
        umma::launch_p1_umma(t.tmW, pa, P.g.N_pad, c.st);
    } else {
        launch_p1_weights(w, static_cast<double*>(P.d_mean.p), static_cast<double*>(P.d_sdinv.p),
                          static_cast<double*>(t.z.p), M, 0, c.st);
        if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
        launch_p1(P.g, w, nullptr, y, c.st);
    }
    if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
}

// Phase 2 of V-tile ti from the sketch y: its digits, then
// accum += the guarded per-SNP updates over this image's SNPs.
void plan_enqueue_phase2(Context& c, GwPlan& pl, size_t ti, const double* y, cudaEvent_t* ev,
                         int& e, cudaEvent_t chk_ev = nullptr) {
    Prepared& P = *pl.P;
    const int64_t M = P.g.M, K = pl.K;
    GwPlan::Tile& t = *pl.tiles[ti];
    if (pl.umma) {
        const int nc = umma::ncolp_for(t.V);
        int* colsum = P.has_complete ? static_cast<int*>(pl.colsum.p) : nullptr;
        umma::launch_quantize_y4(y, P.g.N, P.g.N_pad, (int)K, t.V, nc,
                                 static_cast<int8_t*>(pl.yq.p), static_cast<double*>(pl.ycs.p),
                                 c.st, colsum);
        if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
        umma::P2UArgs u;
        u.K = (int)K;
        u.V = t.V;
        u.ncolp = nc;
        u.bins_per_cta = umma::p2_bins_per_cta_grouped(nc, (int)K);
        u.ngroups = (u.bins_per_cta * nc + 255) / 256;
        u.box_rows = std::min(256, u.bins_per_cta * nc);
        u.nkt = (int)(P.g.N_pad / 128);
        u.M = M;
        u.j0 = 0;
        u.j1 = M;
        u.out_row0 = 0;
        u.colscale = static_cast<double*>(pl.ycs.p);
        u.mean = static_cast<double*>(P.d_mean.p);
        u.sdinv = static_cast<double*>(P.d_sdinv.p);
        u.left_scale = static_cast<double*>(pl.lscale.p);
        u.accum = static_cast<double*>(pl.accum.p);
        u.mc = pl.with_mc ? static_cast<double*>(pl.mc.p) : nullptr;
        u.guard_counts = static_cast<unsigned long long*>(pl.guards.p);
        u.extreme_warn = extreme_warn_env();
        u.drop_extreme = drop_extreme_env();
        u.status = static_cast<unsigned*>(pl.status.p);
        if (colsum) {
            u.snp_missing = static_cast<const uint8_t*>(P.d_missing.p);
            u.colsum = colsum;
        }
        u.yq = static_cast<const int8_t*>(pl.yq.p);
        u.yq_cols = K * nc;
        u.accum_elems = M * K;
        static const bool grid_order = [] {
            const char* e = std::getenv("LDS_P2_GRID_ORDER");
            return e && std::atoi(e) != 0;
        }();
        for (size_t q = 0; q < pl.work_nb.size() && !grid_order; ++q)
            if (pl.work_nb[q] == u.bins_per_cta) {
                u.work = static_cast<const int2*>(pl.work[q]->p);
                u.n_work = pl.n_work[q];
            }
        int v0 = 0;
        for (size_t q = 0; q < ti; ++q) v0 += pl.tiles[q]->V;
        if (pl.check) {
            u.chk = static_cast<unsigned long long*>(pl.chk_lhs.p);
            u.chk_v0 = v0;
        }
        umma::launch_p2_umma(pl.tmA, u, c.st);
        if (pl.check) {
            if (chk_ev) ck(cudaEventRecord(chk_ev, c.st), "event");
            auto* ub = static_cast<unsigned long long*>(pl.chk_u.p);
            launch_check_u(static_cast<const int8_t*>(pl.yq.p), K * nc, nc, (int)K, t.V, v0, 1,
                           P.g.N_pad, ub, c.st);
            launch_check_rhs(P.g.codes, P.g.nbp, static_cast<const int4*>(pl.chk_tiles.p),
                             pl.chk_ntiles, (int)K, ub, P.g.N_pad,
                             static_cast<unsigned long long*>(pl.chk_rhs.p), c.st);
        }
        if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
        return;
    }
    launch_quantize_y(y, P.g.N, P.g.N_pad, (int)K, t.V, t.Vp, pl.S, static_cast<int8_t*>(pl.yq.p),
                      static_cast<double*>(pl.ycs.p), c.st);
    if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
    P2Args a;
    a.K = (int)K;
    a.V = t.V;
    a.Vp = t.Vp;
    a.S = pl.S;
    a.j0 = 0;
    a.j1 = M;
    a.out_row0 = 0;
    a.Yq = static_cast<int8_t*>(pl.yq.p);
    a.colscale = static_cast<double*>(pl.ycs.p);
    a.mean = static_cast<double*>(P.d_mean.p);
    a.sdinv = static_cast<double*>(P.d_sdinv.p);
    a.left_scale = static_cast<double*>(pl.lscale.p);
    a.accum = static_cast<double*>(pl.accum.p);
    a.mc = pl.with_mc ? static_cast<double*>(pl.mc.p) : nullptr;
    a.guard_counts = static_cast<unsigned long long*>(pl.guards.p);
    a.extreme_warn = extreme_warn_env();
    a.drop_extreme = drop_extreme_env();
    launch_p2(P.g, a, c.st);
    if (ev) ck(cudaEventRecord(ev[e++], c.st), "event");
}

void plan_execute(Context& c, GwPlan& pl) {
    plan_zero(c, pl);
    const bool tm = pl.pending < GwPlan::kMaxTimed;
    cudaEvent_t* ev = nullptr;
    if (tm) {
        if ((int)pl.evsets.size() <= pl.pending) {
            std::vector<cudaEvent_t> set(1 + 4 * pl.tiles.size());
            for (auto& x : set) ck(cudaEventCreate(&x), "event");
            pl.evsets.push_back(std::move(set));
        }
        ev = pl.evsets[(size_t)pl.pending].data();
        if (pl.check) {
            while ((int)pl.chk_evsets.size() <= pl.pending) {
                std::vector<cudaEvent_t> set(pl.tiles.size());
                for (auto& x : set) ck(cudaEventCreate(&x), "event");
                pl.chk_evsets.push_back(std::move(set));
            }
        }
    }
    pl.executed = 1;
    int e = 0;
    if (tm) ck(cudaEventRecord(ev[e++], c.st), "event");
    double* y = static_cast<double*>(pl.y.p);
    for (size_t ti = 0; ti < pl.tiles.size(); ++ti) {
        plan_enqueue_phase1(c, pl, ti, y, ev, e);
        plan_enqueue_phase2(c, pl, ti, y, ev, e,
                            (tm && pl.check) ? pl.chk_evsets[(size_t)pl.pending][ti] : nullptr);
    }
    if (tm) ++pl.pending;
    ck(cudaGetLastError(), "launch");
}

// Mean per-execute kernel times over the executes since the last call.
void plan_kernel_times(GwPlan& pl) {
    if (pl.pending == 0) return;
    for (double& x : pl.kernel_ms) x = 0.0;
    pl.check_ms = 0.0;
    const size_t nt = pl.tiles.size();
    for (int p = 0; p < pl.pending; ++p) {
        const std::vector<cudaEvent_t>& ev = pl.evsets[(size_t)p];
        ck(cudaEventSynchronize(ev[4 * nt]), "event sync");
        for (size_t t = 0; t < nt; ++t)
            for (int k = 0; k < 4; ++k) {
                float ms = 0.f;
                // with checks, phase 2 ends at the check event and the check
                // kernels run from there to the tile's last event
                const cudaEvent_t end = (k == 3 && pl.check && pl.umma)
                                            ? pl.chk_evsets[(size_t)p][t] : ev[4 * t + k + 1];
                ck(cudaEventElapsedTime(&ms, ev[4 * t + k], end), "elapsed");
                pl.kernel_ms[k] += ms;
                if (end != ev[4 * t + k + 1]) {
                    ck(cudaEventElapsedTime(&ms, end, ev[4 * t + k + 1]), "elapsed");
                    pl.check_ms += ms;
                }
            }
    }
    for (double& x : pl.kernel_ms) x /= (double)pl.pending;
    pl.check_ms /= (double)pl.pending;
    pl.pending = 0;
}

void plan_results(Context& c, GwPlan& pl, double* ldscore, double* meansq_out, double* inv_out,
                  double* mc_agg, double* mc_snp) {
    const int64_t M = pl.P->g.M, K = pl.K, N = pl.P->g.N;
    std::vector<double> acc((size_t)(M * K));
    d2h(acc.data(), static_cast<double*>(pl.accum.p), acc.size(), c.st);
    std::vector<double> mcv;
    if (pl.with_mc) {
        mcv.resize((size_t)(M * K));
        d2h(mcv.data(), static_cast<double*>(pl.mc.p), mcv.size(), c.st);
    }
    ck(cudaStreamSynchronize(c.st), "results");
    if (pl.umma) {
        unsigned st = 0;
        d2h(&st, static_cast<unsigned*>(pl.status.p), 1, c.st);
        ck(cudaStreamSynchronize(c.st), "status");
        if (st) fail(LDS_ERR_CUDA, "phase-2 tensor-core pipeline wait timed out (code %u)", st);
    }
    plan_kernel_times(pl);
    {
        unsigned long long h[2] = {0, 0};
        d2h(h, static_cast<unsigned long long*>(pl.guards.p), 2, c.st);
        ck(cudaStreamSynchronize(c.st), "guards");
        if (h[0] || h[1])
            std::fprintf(stderr,
                         "[phase2-warning] accum: dropped %llu non-finite and %llu extreme "
                         "LD-score updates; inspect this run before using it.\n", h[0], h[1]);
    }
    if (meansq_out) std::memcpy(meansq_out, acc.data(), sizeof(double) * acc.size());
    if (inv_out) std::memcpy(inv_out, pl.inv.data(), sizeof(double) * (size_t)M);
    // Finalize: / nvecs, minus M_k / (N - ddof) (gw_ldscore.py:2197, :2220-2222).
    const double nd = (double)(N - pl.P->ddof);
    if (ldscore)
        for (int64_t j = 0; j < M; ++j)
            for (int64_t k = 0; k < K; ++k)
                ldscore[j * K + k] = acc[(size_t)(j * K + k)] / (double)pl.nvecs - pl.Mk[(size_t)k] / nd;
    if (pl.with_mc) {
        if (mc_agg)
            for (int64_t k = 0; k < K; ++k) {
                double agg = 0.0;
                for (int64_t j = 0; j < M; ++j) agg += mcv[(size_t)(j * K + k)];
                mc_agg[k] = agg;
            }
        if (mc_snp) std::memcpy(mc_snp, mcv.data(), sizeof(double) * mcv.size());
    }
}

// ---------------------------------------------------------------------------
// Windowed estimates: SNP windows (a contiguous partition, window w = SNPs
// [ws[w], ws[w+1])) are independent genome-wide problems on their SNPs.  Each
// window draws its own probes (root seed window_seed(root, w), blocks of
// `step` SNPs counted from the window start), so window w's LD scores equal
// the genome-wide estimate on the window's sub-fileset with that seed.
// (window, bin) pairs become phase-1 super-bins; phase 2 runs over a tile
// table covering all windows of a batch.  Batches bound the sketch memory.
// ---------------------------------------------------------------------------
uint64_t window_seed(uint64_t root, int64_t w) {
    return mix64(root ^ mix64(0x77696e646f77ULL + (uint64_t)w));
}

struct WinPlan {
    std::shared_ptr<Prepared> P;
    int64_t K = 0, W = 0;
    int nvecs = 0, with_mc = 0;
    std::vector<int> vt;
    std::vector<int64_t> ws;            // W+1 window starts
    std::vector<int32_t> win_of;        // SNP -> window
    std::vector<double> inv, Mkw;       // Mkw[w*K + k]
    struct Batch {
        int64_t w0 = 0, w1 = 0, ksup = 0, lmax = 0;
        Csr csr;
        DevBuf rowind, sc, binoff, tiles;
        int64_t ntiles = 0;                // 128-SNP tiles
        // Phase-2 CTA order per bins-per-CTA value work_nb[i]: window by
        // window, chunks of kWorkBinChunk bin groups, the window's tiles, the
        // chunk's bin groups (a tile's packed codes and a (window, bin)
        // sketch stay in L2 while the CTAs that share them run).
        std::vector<int> work_nb;
        std::vector<std::unique_ptr<DevBuf>> work;
        std::vector<int64_t> n_work;
        std::vector<int64_t> tile_begin;   // first tile of each window, and the tile count
    };
    std::vector<Batch> batches;
    std::vector<DevBuf> z;              // per V-tile, M x V FP64 probes
    DevBuf y, ycs, yshift, wcs, accum, mc, lscale, guards, status;
    DevBuf colsum;                      // sketch digit column sums (images with complete tiles)
    std::shared_ptr<DevBuf> yq, wq;     // shared context workspaces (Context::ws)
    // Optional outputs for the control variate (lds_win_plan_set_cv): per-V-tile
    // meansq slices, near-field sums C and known means mu, neighbour products.
    int split = 0, cv_D = 0;
    // Tiling chosen for this plan (lds_win_plan_set_tiling): phase-1 super-bins
    // per CTA (0: default).
    int p1_spc = 0;
    // Phase-2 CTA shape and order (lds_win_plan_set_p2_bins / _set_p2_order):
    // bins per CTA (0: p2_bins_per_cta_grouped) and bins per chunk of the
    // window-major work order (0: grid order).
    int p2_nb = 0, p2_chunk = 4;
    int p2_bins(int ncolp) const {
        return p2_nb > 0 ? (int)std::min<int64_t>(p2_nb, K)
                         : umma::p2_bins_per_cta_grouped(ncolp, (int)K);
    }
    DevBuf annot_d, winof_d, sqrt_ls, xx, band_cnt, cvC, cvMu;
    DevBuf mkw_d, ld_d, ms_d;           // finalize inputs and outputs
    cudaEvent_t cv_ev[2] = {nullptr, nullptr};
    double cv_ms = 0.0;
    CUtensorMap tmA;
    std::vector<cudaEvent_t> ev;        // start, after phase 1 of each launch group, end
    // weights, phase 1, digits, phase 2 and (with checks) product checks
    double kernel_ms[5] = {0, 0, 0, 0, 0};
    int pending = 0;
    // Product checksums (lds_win_plan_set_checks): lhs from the phase-2
    // epilogue, rhs from the CUDA-core pass (lds_check.cu), 2 per SNP; u per
    // window of the largest batch.
    int check = 0;
    DevBuf chk_lhs, chk_rhs, chk_u;
    int ev_per() const { return check ? 5 : 4; }
    cudaGraphExec_t graph = nullptr;
    unsigned long long graph_kernels = 0;  // kernel nodes in the captured graph
    // Output slices: with `split`, probes [0, half) and [half, nvecs) of every
    // (SNP, bin) sum go to two slices (two independent halves of the probes).
    int ntiles_out() const { return split ? 2 : 1; }
    int half() const { return (nvecs + 1) / 2; }
    // Probe range of V-tile ti: [voff(ti), voff(ti) + vt[ti]).
    int voff(size_t ti) const {
        int o = 0;
        for (size_t u = 0; u < ti; ++u) o += vt[u];
        return o;
    }
    int split_local(size_t ti) const { return std::min(std::max(half() - voff(ti), 0), vt[ti]); }
    ~WinPlan() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        for (cudaEvent_t e : cv_ev)
            if (e) cudaEventDestroy(e);
        if (graph) cudaGraphExecDestroy(graph);
    }
};

// A context workspace of at least `bytes` (slot 0 sketch digits, 1 weight digits).
std::shared_ptr<DevBuf> shared_workspace(Context& c, int slot, size_t bytes) {
    PoolScope plain(nullptr, nullptr);  // outlives its plan: ordinary device memory
    std::shared_ptr<DevBuf>& w = c.ws[slot];
    if (!w || w->n < bytes) {
        w.reset();  // plans that captured the old buffer keep it alive
        w = std::make_shared<DevBuf>();
        w->get(bytes);
    }
    return w;
}

// Phase-2 CTA orders of a window batch, one per bins-per-CTA value of the
// V-tiles: window by window, chunks of about p2_chunk bins (whole CTA bin
// groups, at least one), the window's tiles, the chunk's bin groups
// (p2_chunk 0: no order, the grid's).
void build_win_work(Context& c, const WinPlan& pl, WinPlan::Batch& b) {
    const int64_t K = pl.K;
    b.work_nb.clear();
    b.work.clear();
    b.n_work.clear();
    if (pl.p2_chunk <= 0) return;
    for (int V : pl.vt) {
        const int nb = pl.p2_bins(umma::ncolp_for(V));
        if (std::find(b.work_nb.begin(), b.work_nb.end(), nb) != b.work_nb.end()) continue;
        const int groups = (int)((K + nb - 1) / nb);
        const int chunk = std::max(1, pl.p2_chunk / nb);
        std::vector<int2> order;
        for (size_t w = 0; w + 1 < b.tile_begin.size(); ++w)
            for (int g0 = 0; g0 < groups; g0 += chunk)
                for (int64_t t = b.tile_begin[w]; t < b.tile_begin[w + 1]; ++t)
                    for (int g = g0; g < std::min(groups, g0 + chunk); ++g)
                        order.push_back(make_int2((int)t, g));
        auto buf = std::make_unique<DevBuf>();
        h2d(buf->as<int2>(order.size()), order.data(), order.size(), c.st);
        b.work_nb.push_back(nb);
        b.work.push_back(std::move(buf));
        b.n_work.push_back((int64_t)order.size());
    }
}

std::map<int64_t, std::unique_ptr<WinPlan>>& win_table() {
    static std::map<int64_t, std::unique_ptr<WinPlan>> t;
    return t;
}

std::unique_ptr<WinPlan> win_plan_create(Context& c, std::shared_ptr<Prepared> P,
                                         const double* annot, int64_t K, const int64_t* ws,
                                         int64_t W, int nvecs, int step, int vtile, uint64_t seed,
                                         int dist, double eps, int as_float, int with_mc,
                                         double batch_gb, int64_t w_base = 0) {
    const int64_t M = P->g.M, N = P->g.N, Np = P->g.N_pad;
    if (nvecs <= 0 || step <= 0 || K <= 0 || W <= 0) fail(LDS_ERR_ARG, "invalid sizes");
    if (ws[0] != 0 || ws[W] != M) fail(LDS_ERR_ARG, "windows must partition [0, M)");
    for (int64_t w = 0; w < W; ++w)
        if (ws[w + 1] <= ws[w]) fail(LDS_ERR_ARG, "window starts must increase");
    if (c.slices != 4 || p2_impl() != 1)
        fail(LDS_ERR_ARG, "windowed estimates need the tcgen05 kernels with 4 digits");
    auto pl = std::make_unique<WinPlan>();
    pl->P = P;
    pl->K = K;
    pl->W = W;
    pl->nvecs = nvecs;
    pl->with_mc = with_mc;
    pl->ws.assign(ws, ws + W + 1);
    pl->win_of.resize((size_t)M);
    for (int64_t w = 0; w < W; ++w)
        for (int64_t j = ws[w]; j < ws[w + 1]; ++j) pl->win_of[(size_t)j] = (int32_t)w;
    {
        int width = std::min(nvecs, vtile > 0 ? vtile : nvecs);
        if (width >= 64) width = std::max(64, (width / 64) * 64);
        for (int s = 0; s < nvecs; s += width) pl->vt.push_back(std::min(width, nvecs - s));
    }
    const int vmax = *std::max_element(pl->vt.begin(), pl->vt.end());
    const int ncmax = umma::ncolp_for(vmax);
    pl->inv.resize((size_t)M);
    for (int64_t j = 0; j < M; ++j)
        pl->inv[(size_t)j] =
            as_float ? (double)inv_resvar<float>(*P, j, eps) : inv_resvar<double>(*P, j, eps);
    // Per-window annotation totals, summed in SNP order within each window
    // (windows in parallel on host threads).
    pl->Mkw.assign((size_t)(W * K), 0.0);
    const unsigned hw_win = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    auto par_windows = [&](const std::function<void(int64_t)>& body) {
        std::vector<std::thread> th;
        std::atomic<int64_t> next{0};
        for (unsigned t = 0; t < hw_win; ++t)
            th.emplace_back([&] {
                for (int64_t w; (w = next.fetch_add(1)) < W;) body(w);
            });
        for (auto& x : th) x.join();
    };
    par_windows([&](int64_t w) {
        double* mk = &pl->Mkw[(size_t)(w * K)];
        for (int64_t j = ws[w]; j < ws[w + 1]; ++j)
            for (int64_t k = 0; k < K; ++k) mk[k] += annot[j * K + k];
    });
    const double denom = std::max(1.0, (double)(N - P->ddof + 1) - 1.0);
    const double inv_denom2 = 1.0 / (denom * denom);
    std::vector<double> ls((size_t)M);
    for (int64_t j = 0; j < M; ++j) {
        const double v = pl->inv[(size_t)j];
        ls[(size_t)j] = (std::isfinite(v) && v > 0.0) ? v * v * inv_denom2 : 0.0;
    }
    h2d(pl->lscale.as<double>((size_t)M), ls.data(), (size_t)M, c.st);
    h2d(pl->winof_d.as<int32_t>((size_t)M), pl->win_of.data(), (size_t)M, c.st);
    h2d(pl->mkw_d.as<double>(pl->Mkw.size()), pl->Mkw.data(), pl->Mkw.size(), c.st);
    // Window batches: the sketch digits of a batch stay under batch_gb.
    const double per_window = (double)Np * (double)K * umma::ncolp_for(vmax);
    const int64_t wb = std::max<int64_t>(1, (int64_t)(batch_gb * 1e9 / per_window));
    std::vector<float> annot_f, inv_f;
    if (as_float) {
        annot_f.assign(annot, annot + M * K);
        inv_f.resize((size_t)M);
        for (int64_t j = 0; j < M; ++j) inv_f[(size_t)j] = (float)pl->inv[(size_t)j];
    }
    // Member lists of every (window, bin), built on host threads.
    std::vector<Csr> parts((size_t)W);
    par_windows([&](int64_t w) {
        const int64_t a0 = ws[w], L = ws[w + 1] - ws[w];
        const uint8_t* cst = P->constant.data();
        parts[(size_t)w] = as_float
            ? build_csr<float>(annot_f.data() + a0 * K, inv_f.data() + a0, L, K, a0, 16, 4, 128, cst)
            : build_csr<double>(annot + a0 * K, pl->inv.data() + a0, L, K, a0, 16, 4, 128, cst);
    });
    int64_t max_ksup = 0, max_wq = 0;
    for (int64_t w0 = 0; w0 < W; w0 += wb) {
        WinPlan::Batch b;
        b.w0 = w0;
        b.w1 = std::min(W, w0 + wb);
        b.ksup = (b.w1 - b.w0) * K;
        // Super-bin CSR: super-bin (w - w0)*K + k lists the window's members of bin k.
        Csr cs;
        cs.bin_off.assign((size_t)b.ksup + 1, 0);
        cs.nnz.assign((size_t)b.ksup, 0);
        std::vector<int32_t> ri;
        std::vector<double> scv;
        int64_t off = 0;
        for (int64_t w = b.w0; w < b.w1; ++w) {
            const Csr& part = parts[(size_t)w];
            for (int64_t k = 0; k < K; ++k) {
                const int64_t sbk = (w - b.w0) * K + k;
                cs.bin_off[(size_t)sbk] = off;
                cs.nnz[(size_t)sbk] = part.nnz[(size_t)k];
                const int64_t p0 = part.bin_off[(size_t)k], p1 = part.bin_off[(size_t)k + 1];
                ri.insert(ri.end(), part.rowind.begin() + p0, part.rowind.begin() + p1);
                scv.insert(scv.end(), part.sc.begin() + p0, part.sc.begin() + p1);
                off += p1 - p0;
                b.lmax = std::max(b.lmax, p1 - p0);
            }
        }
        cs.bin_off[(size_t)b.ksup] = off;
        b.lmax = std::max<int64_t>(b.lmax, 128);
        const size_t nm = std::max<size_t>(ri.size(), 1);
        h2d(b.rowind.as<int32_t>(nm), ri.data(), ri.size(), c.st);
        h2d(b.sc.as<double>(nm), scv.data(), scv.size(), c.st);
        h2d(b.binoff.as<int64_t>(cs.bin_off.size()), cs.bin_off.data(), cs.bin_off.size(), c.st);
        std::vector<int4> tiles;
        std::vector<int64_t> tile_begin;   // first tile of each window of the batch
        for (int64_t w = b.w0; w < b.w1; ++w) {
            tile_begin.push_back((int64_t)tiles.size());
            for (int64_t j = ws[w]; j < ws[w + 1]; j += 128)
                tiles.push_back(make_int4((int)j, (int)ws[w + 1], (int)((w - b.w0) * K), 0));
        }
        tile_begin.push_back((int64_t)tiles.size());
        b.ntiles = (int64_t)tiles.size();
        h2d(b.tiles.as<int4>(tiles.size()), tiles.data(), tiles.size(), c.st);
        b.tile_begin = std::move(tile_begin);
        build_win_work(c, *pl, b);
        ck(cudaStreamSynchronize(c.st), "window batch upload");
        max_ksup = std::max(max_ksup, b.ksup);
        max_wq = std::max(max_wq, b.ksup * 2 * ncmax * b.lmax);
        b.csr.nnz = cs.nnz;
        pl->batches.push_back(std::move(b));
    }
    // Probes: per window, blocks counted from the window start.
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::pair<int64_t, int64_t>> units;  // (window, relative block start)
    for (int64_t w = 0; w < W; ++w)
        for (int64_t s = 0; s < ws[w + 1] - ws[w]; s += step) units.push_back({w, s});
    int v0 = 0;
    for (int V : pl->vt) {
        pl->z.emplace_back();
        double* dZ = pl->z.back().as<double>((size_t)(M * V));
        if (dist == LDS_DIST_RADEMACHER) {
            std::vector<ProbeUnit> pu(units.size());
            for (size_t u = 0; u < units.size(); ++u) {
                const int64_t w = units[u].first, s = units[u].second;
                pu[u] = {ws[w] + s, (int32_t)std::min<int64_t>(step, ws[w + 1] - ws[w] - s), 0,
                         probe_seed(window_seed(seed, w_base + w), (int)s, v0)};
            }
            device_rademacher(c, pu, V, dZ, M);
            v0 += V;
            continue;
        }
        std::vector<double> Z((size_t)(M * V));
        std::vector<std::thread> th;
        std::atomic<size_t> next{0};
        for (unsigned t = 0; t < hw; ++t)
            th.emplace_back([&] {
                for (size_t u; (u = next.fetch_add(1)) < units.size();) {
                    const int64_t w = units[u].first, s = units[u].second;
                    const int64_t a0 = ws[w];
                    const int L = (int)std::min<int64_t>(step, ws[w + 1] - a0 - s);
                    const uint64_t rw = window_seed(seed, w_base + w);
                    if (as_float) make_probes<float>(rw, (int)s, v0, L, V, dist, &Z[(size_t)(a0 + s)], M);
                    else make_probes<double>(rw, (int)s, v0, L, V, dist, &Z[(size_t)(a0 + s)], M);
                }
            });
        for (auto& x : th) x.join();
        h2d(dZ, Z.data(), Z.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "probe upload");
        v0 += V;
    }
    pl->yq = shared_workspace(c, 0, (size_t)(max_ksup * ncmax * Np));
    pl->ycs.as<double>((size_t)(max_ksup * vmax));
    pl->yshift.as<int>((size_t)(max_ksup * vmax));
    if (P->has_complete) pl->colsum.as<int>((size_t)(max_ksup * ncmax));
    pl->wq = shared_workspace(c, 1, (size_t)std::max<int64_t>(max_wq, 16));
    pl->wcs.as<double>((size_t)(max_ksup * vmax));
    pl->accum.as<double>((size_t)(M * K));
    if (with_mc) pl->mc.as<double>((size_t)(M * K));
    pl->guards.as<unsigned long long>(2);
    ck(cudaMemsetAsync(pl->status.as<unsigned>(1), 0, 4, c.st), "memset");
    pl->tmA = make_map_2d(P->g.codes, (uint64_t)P->g.nbp, (uint64_t)P->g.M_pad, (uint64_t)P->g.nbp,
                          32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
    pl->ev.resize(1 + 4 * pl->vt.size() * pl->batches.size());
    for (auto& e : pl->ev) ck(cudaEventCreate(&e), "event");
    umma::prepare_p1_umma();
    umma::prepare_p2_umma();
    ck(cudaStreamSynchronize(c.st), "window plan");
    return pl;
}

// Enqueue one windowed estimate (all V-tiles, all batches).
void win_enqueue(Context& c, WinPlan& pl) {
    Prepared& P = *pl.P;
    const int64_t M = P.g.M, K = pl.K, Np = P.g.N_pad;
    const size_t MK = (size_t)(M * K), nout = MK * (size_t)pl.ntiles_out();
    ck(cudaMemsetAsync(pl.accum.p, 0, sizeof(double) * nout, c.st), "memset");
    if (pl.with_mc) ck(cudaMemsetAsync(pl.mc.p, 0, sizeof(double) * MK, c.st), "memset");
    ck(cudaMemsetAsync(pl.guards.p, 0, 16, c.st), "memset");
    if (pl.check) {
        ck(cudaMemsetAsync(pl.chk_lhs.p, 0, sizeof(unsigned long long) * 2 * (size_t)M, c.st), "memset");
        ck(cudaMemsetAsync(pl.chk_rhs.p, 0, sizeof(unsigned long long) * 2 * (size_t)M, c.st), "memset");
    }
    if (pl.cv_D > 0) {
        // Near-field control variate sums: inputs are static (probes, products),
        // so they run first, timed by their own event pair.
        ck(cudaEventRecordWithFlags(pl.cv_ev[0], c.st, cudaEventRecordExternal), "event");
        ck(cudaMemsetAsync(pl.cvC.p, 0, sizeof(double) * nout, c.st), "memset");
        for (size_t ti = 0; ti < pl.vt.size(); ++ti) {
            CvNearArgs a;
            a.M = M;
            a.K = (int)K;
            a.V = pl.vt[ti];
            a.z = static_cast<double*>(pl.z[ti].p);
            a.z_ld = M;
            a.annot = static_cast<double*>(pl.annot_d.p);
            a.win_of = static_cast<int32_t*>(pl.winof_d.p);
            a.sqrt_ls = static_cast<double*>(pl.sqrt_ls.p);
            a.xx = static_cast<double*>(pl.xx.p);
            a.C = static_cast<double*>(pl.cvC.p);
            a.mu = ti == 0 ? static_cast<double*>(pl.cvMu.p) : nullptr;
            if (pl.split) {
                a.C2 = static_cast<double*>(pl.cvC.p) + MK;
                a.split_v = pl.split_local(ti);
            }
            launch_cv_near(a, pl.cv_D, c.st);
        }
        ck(cudaEventRecordWithFlags(pl.cv_ev[1], c.st, cudaEventRecordExternal), "event");
    }
    int e = 0;
    ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
    for (size_t ti = 0; ti < pl.vt.size(); ++ti) {
        const int V = pl.vt[ti];
        const int nc = umma::ncolp_for(V);
        // Phase 1 writes every digit row of every super-bin of a batch, the
        // padding rows 4V..ncolp included (as zeros), so the buffer needs no clearing.
        for (auto& b : pl.batches) {
            umma::P1UWeights uw;
            uw.K = (int)b.ksup;
            uw.V = V;
            uw.ncolp = nc;
            uw.lmax = b.lmax;
            uw.rowind = static_cast<int32_t*>(b.rowind.p);
            uw.sc = static_cast<double*>(b.sc.p);
            uw.bin_off = static_cast<int64_t*>(b.binoff.p);
            uw.wq = static_cast<int8_t*>(pl.wq->p);
            uw.colscale = static_cast<double*>(pl.wcs.p);
            uw.ycolscale = static_cast<double*>(pl.ycs.p);
            uw.yshift = static_cast<int*>(pl.yshift.p);
            const size_t wbytes = (size_t)(b.ksup * 2 * nc) * (size_t)b.lmax;
            ck(cudaMemsetAsync(pl.wq->p, 0, wbytes, c.st), "memset weights");
            umma::launch_p1_weights4(uw, static_cast<double*>(P.d_mean.p),
                                     static_cast<double*>(P.d_sdinv.p),
                                     static_cast<double*>(pl.z[ti].p), M, c.st);
            ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
            const CUtensorMap tmW =
                make_map_2d(pl.wq->p, (uint64_t)b.lmax, (uint64_t)(b.ksup * 2 * nc), (uint64_t)b.lmax,
                            128, (uint32_t)std::min(256, nc), CU_TENSOR_MAP_SWIZZLE_128B);
            umma::P1UArgs pa;
            pa.K = (int)b.ksup;
            pa.V = V;
            pa.ncolp = nc;
            pa.ngroups = (nc + 255) / 256;
            pa.box_rows = std::min(256, nc);
            pa.nbp = P.g.nbp;
            pa.N_pad = Np;
            pa.bin_off = uw.bin_off;
            pa.rowind = uw.rowind;
            pa.codes = P.g.codes;
            pa.colscale = uw.colscale;
            pa.Y = nullptr;
            pa.status = static_cast<unsigned*>(pl.status.p);
            static const int spc = [] {
                const char* e = std::getenv("LDS_P1_SB_PER_CTA");
                const int v = e ? std::atoi(e) : 0;
                return v > 0 ? v : 8;
            }();
            pa.sb_per_cta = pl.p1_spc > 0 ? pl.p1_spc : spc;
            pa.yq = static_cast<int8_t*>(pl.yq->p);
            pa.ycolscale = static_cast<double*>(pl.ycs.p);
            pa.yshift = static_cast<int*>(pl.yshift.p);
            pa.m_pad = P.g.M_pad;
            umma::launch_p1_umma(tmW, pa, Np, c.st);
            ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
            // (sketch digits were written by phase 1's epilogue; their column
            // sums stand in for the O plane of tiles without missing calls)
            int* colsum = P.has_complete ? static_cast<int*>(pl.colsum.p) : nullptr;
            if (colsum)
                umma::launch_digit_colsum(static_cast<const int8_t*>(pl.yq->p), b.ksup * nc, Np,
                                          colsum, c.st);
            ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
            const int nb = pl.p2_bins(nc);
            umma::P2UArgs u;
            u.yq = static_cast<const int8_t*>(pl.yq->p);
            u.yq_cols = b.ksup * nc;
            u.K = (int)K;
            u.V = V;
            u.ncolp = nc;
            u.bins_per_cta = nb;
            u.ngroups = (nb * nc + 255) / 256;
            u.box_rows = std::min(256, nb * nc);
            u.nkt = (int)(Np / 128);
            u.M = M;
            u.j0 = 0;
            u.j1 = b.ntiles;  // number of tiles (tile-table mode)
            u.out_row0 = 0;
            u.colscale = static_cast<double*>(pl.ycs.p);
            u.mean = static_cast<double*>(P.d_mean.p);
            u.sdinv = static_cast<double*>(P.d_sdinv.p);
            u.left_scale = static_cast<double*>(pl.lscale.p);
            u.accum = static_cast<double*>(pl.accum.p);
            if (pl.split) {
                u.accum2 = static_cast<double*>(pl.accum.p) + MK;
                u.split_v = pl.split_local(ti);
            }
            u.mc = pl.with_mc ? static_cast<double*>(pl.mc.p) : nullptr;
            u.guard_counts = static_cast<unsigned long long*>(pl.guards.p);
            u.extreme_warn = extreme_warn_env();
            u.drop_extreme = drop_extreme_env();
            u.status = static_cast<unsigned*>(pl.status.p);
            if (colsum) {
                u.snp_missing = static_cast<const uint8_t*>(P.d_missing.p);
                u.colsum = colsum;
            }
            u.accum_elems = (int64_t)MK;
            u.tiles = static_cast<int4*>(b.tiles.p);
            static const bool grid_order = [] {
                const char* e = std::getenv("LDS_P2_GRID_ORDER");
                return e && std::atoi(e) != 0;
            }();
            for (size_t q = 0; q < b.work_nb.size() && !grid_order; ++q)
                if (b.work_nb[q] == nb) {
                    u.work = static_cast<const int2*>(b.work[q]->p);
                    u.n_work = b.n_work[q];
                }
            if (pl.check) {
                u.chk = static_cast<unsigned long long*>(pl.chk_lhs.p);
                u.chk_v0 = pl.voff(ti);
            }
            umma::launch_p2_umma(pl.tmA, u, c.st);
            ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
            if (pl.check) {
                // the same products, recomputed on the CUDA cores before the
                // next batch's phase 1 overwrites the sketch digits
                auto* ub = static_cast<unsigned long long*>(pl.chk_u.p);
                launch_check_u(static_cast<const int8_t*>(pl.yq->p), b.ksup * nc, nc, (int)K, V,
                               pl.voff(ti), b.w1 - b.w0, Np, ub, c.st);
                launch_check_rhs(P.g.codes, P.g.nbp, static_cast<const int4*>(b.tiles.p), b.ntiles,
                                 (int)K, ub, Np, static_cast<unsigned long long*>(pl.chk_rhs.p),
                                 c.st);
                ck(cudaEventRecordWithFlags(pl.ev[(size_t)e++], c.st, cudaEventRecordExternal), "event");
            }
        }
    }
    ck(cudaGetLastError(), "launch");
}

// Execute: the first call runs eagerly (kernel attributes, tensor maps) and
// then captures the whole estimate into a CUDA graph; later calls launch it.
void win_execute(Context& c, WinPlan& pl) {
    if (!pl.graph) {
        cudaGraph_t g = nullptr;
        const unsigned long long l0 = g_launches.load();
        ck(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal), "capture");
        try {
            win_enqueue(c, pl);
        } catch (...) {
            cudaStreamEndCapture(c.st, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        ck(cudaStreamEndCapture(c.st, &g), "capture end");
        ck(cudaGraphInstantiate(&pl.graph, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        // Captured launches did not run; count them when the graph does.
        pl.graph_kernels = g_launches.load() - l0;
        g_launches.fetch_sub(pl.graph_kernels);
    }
    ck(cudaGraphLaunch(pl.graph, c.st), "graph launch");
    g_launches.fetch_add(pl.graph_kernels);
    pl.pending = 1;
}

void win_times(WinPlan& pl) {
    if (!pl.pending) return;
    ck(cudaEventSynchronize(pl.ev.back()), "event sync");
    for (double& x : pl.kernel_ms) x = 0.0;
    if (pl.cv_D > 0) {
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, pl.cv_ev[0], pl.cv_ev[1]), "elapsed");
        pl.cv_ms = ms;
    }
    for (size_t i = 0; i + 1 < pl.ev.size(); ++i) {
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, pl.ev[i], pl.ev[i + 1]), "elapsed");
        // event order per (V-tile, batch): weights, phase 1, digits, phase 2
        // and, with checks, the product check
        pl.kernel_ms[i % (size_t)pl.ev_per()] += ms;
    }
    pl.pending = 0;
}

void win_results(Context& c, WinPlan& pl, double* ldscore, double* meansq_out, double* inv_out,
                 double* mc_snp) {
    const int64_t M = pl.P->g.M, K = pl.K, N = pl.P->g.N;
    const size_t MK = (size_t)(M * K);
    // Per-V-tile slices (control-variate plans) add up to the plain sums; the
    // finalize runs on the device and the outputs go straight to the caller.
    const double nd = (double)(N - pl.P->ddof);
    double* dld = pl.ld_d.as<double>(MK);
    double* dms = pl.ms_d.as<double>(MK);
    launch_win_finalize(static_cast<double*>(pl.accum.p), pl.ntiles_out(), M, (int)K,
                        (double)pl.nvecs, nd, static_cast<int32_t*>(pl.winof_d.p),
                        static_cast<double*>(pl.mkw_d.p), dld, dms, c.st);
    ck(cudaGetLastError(), "finalize");
    unsigned st = 0;
    d2h(&st, static_cast<unsigned*>(pl.status.p), 1, c.st);
    ck(cudaStreamSynchronize(c.st), "results");
    if (st) fail(LDS_ERR_CUDA, "tensor-core pipeline wait timed out (code %u)", st);
    win_times(pl);
    if (ldscore) d2h(ldscore, dld, MK, c.st);
    if (meansq_out) d2h(meansq_out, dms, MK, c.st);
    if (pl.with_mc && mc_snp) d2h(mc_snp, static_cast<double*>(pl.mc.p), MK, c.st);
    ck(cudaStreamSynchronize(c.st), "results copy");
    if (inv_out) std::memcpy(inv_out, pl.inv.data(), sizeof(double) * (size_t)M);
}

// Finalize of a windowed plan on c.st, outputs copied into pinned host memory
// without waiting (the caller synchronizes before reading them).
void win_results_async(Context& c, WinPlan& pl, double* h_ld, double* h_ms, unsigned* h_status) {
    const int64_t M = pl.P->g.M, K = pl.K, N = pl.P->g.N;
    const size_t MK = (size_t)(M * K);
    double* dld = pl.ld_d.as<double>(MK);
    double* dms = pl.ms_d.as<double>(MK);
    launch_win_finalize(static_cast<double*>(pl.accum.p), pl.ntiles_out(), M, (int)K,
                        (double)pl.nvecs, (double)(N - pl.P->ddof),
                        static_cast<int32_t*>(pl.winof_d.p), static_cast<double*>(pl.mkw_d.p),
                        dld, dms, c.st);
    ck(cudaGetLastError(), "finalize");
    d2h(h_status, static_cast<unsigned*>(pl.status.p), 1, c.st);
    d2h(h_ld, dld, MK, c.st);
    if (h_ms) d2h(h_ms, dms, MK, c.st);
}

// Windowed estimate in one call from host BED rows, with the upload streamed:
// the windows are cut into window-aligned chunks of about M / n_chunks SNPs,
// and chunk i+1's upload, repack, per-SNP statistics, residual variances,
// member lists and probe streams (image preparation stream, highest priority)
// run while chunk i's estimate runs on the library stream.  Every chunk is a
// windowed plan over its own image with window seeds counted from the global
// window index (and HWE seeds from the global SNP index), so the scores equal
// those of one plan over the whole image bit for bit.  Nothing is freed while
// estimates are in flight: cudaFree waits for the whole device.
void win_ldscore_impl(const uint8_t* bed_rows, int64_t row_bytes, int64_t n_total, int64_t M,
                      const int64_t* row_sel, int64_t n_sel, const double* annot, int64_t K,
                      const int64_t* ws, int64_t W, int nvecs, int step, int vtile, uint64_t seed,
                      int dist, int ddof, int impute, uint64_t iseed, double eps, int as_float,
                      int n_chunks, int p1_spc, double* ldscore, double* meansq_out,
                      double* inv_out) {
    using clk = std::chrono::steady_clock;
    const auto t_start = clk::now();
    auto ms_since = [&](clk::time_point t) {
        return std::chrono::duration<double, std::milli>(clk::now() - t).count();
    };
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (!bed_rows || !annot || !ws || !ldscore) fail(LDS_ERR_ARG, "null input or output");
    if (row_bytes < (n_total + 3) / 4) fail(LDS_ERR_ARG, "bed_row_bytes smaller than ceil(N/4)");
    if (impute != LDS_IMPUTE_MEAN && impute != LDS_IMPUTE_HWE)
        fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
    if (M <= 0 || K <= 0 || W <= 0) fail(LDS_ERR_ARG, "invalid sizes");
    if (ws[0] != 0 || ws[W] != M) fail(LDS_ERR_ARG, "windows must partition [0, M)");
    for (int64_t w = 0; w < W; ++w)
        if (ws[w + 1] <= ws[w]) fail(LDS_ERR_ARG, "window starts must increase");
    if (n_chunks <= 0) n_chunks = 8;
    // Chunk boundaries: the first window start at or after M*f for f = 1/(4n),
    // 3/(4n), then steps of 1/n.  The two short leading chunks make the one
    // upload nothing overlaps short; each next chunk's set-up (about twice as
    // fast as its estimate) still hides behind the previous chunk's estimate.
    std::vector<int64_t> cw{0};
    for (int i = 1; n_chunks > 1; ++i) {
        const double f = i == 1 ? 0.25 / n_chunks : (i - 1.25) / n_chunks;
        if (f >= 1.0) break;
        const int64_t target = (int64_t)(f * (double)M);
        int64_t w = cw.back() + 1;
        while (w < W && ws[w] < target) ++w;
        if (w < W) cw.push_back(w);
    }
    cw.push_back(W);
    const size_t nc = cw.size() - 1;
    if (!c.st_prep) {
        int lo = 0, hi = 0;
        ck(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priorities");
        ck(cudaStreamCreateWithPriority(&c.st_prep, cudaStreamNonBlocking, hi), "prep stream");
    }
    if (!c.pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = c.device;
        ck(cudaMemPoolCreate(&c.pool, &props), "memory pool");
        uint64_t keep = UINT64_MAX;  // keep the reservation (lds_clear_device_cache trims it)
        ck(cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool attr");
    }
    // Grow the context buffers the chunks share to the largest chunk first, so
    // that no chunk's preparation frees (and waits for) a buffer.
    int64_t maxL = 0, max_units = 0;
    for (size_t i = 0; i < nc; ++i) {
        maxL = std::max(maxL, ws[cw[i + 1]] - ws[cw[i]]);
        int64_t u = 0;
        for (int64_t w = cw[i]; w < cw[i + 1]; ++w) u += (ws[w + 1] - ws[w] + step - 1) / step;
        max_units = std::max(max_units, u);
    }
    c.counts_dev.as<SnpCounts>((size_t)maxL);
    c.raw.as<uint8_t>((size_t)(std::max<int64_t>(
                          1, std::min<int64_t>(maxL, (int64_t)(1LL << 30) / row_bytes)) *
                      row_bytes));
    c.units_dev.as<ProbeUnit>((size_t)std::max<int64_t>(max_units, 1));
    if (row_sel) c.rows_dev.as<int32_t>((size_t)n_sel);
    if (impute == LDS_IMPUTE_HWE) {
        c.hwe_q0.as<double>((size_t)maxL);
        c.hwe_q01.as<double>((size_t)maxL);
        c.hwe_sb.as<uint64_t>((size_t)maxL);
    }
    // One window batch per chunk (a chunk's windows in one phase-1 and one
    // phase-2 launch), within 8..32 GB of sketch digits.
    int64_t max_w = 0;
    for (size_t i = 0; i < nc; ++i) max_w = std::max(max_w, cw[i + 1] - cw[i]);
    int vmax = std::min(nvecs, vtile > 0 ? vtile : nvecs);
    if (vmax >= 64) vmax = std::max(64, (vmax / 64) * 64);
    const double per_window =
        (double)round_up(row_sel ? n_sel : n_total, kSamplePad) * (double)K * umma::ncolp_for(vmax);
    const double chunk_gb = std::min(32.0, std::max(8.0, 1.01 * (double)max_w * per_window / 1e9));
    const size_t MK = (size_t)(M * K);
    const size_t need = sizeof(double) * MK * (meansq_out ? 2 : 1) + sizeof(unsigned) * nc;
    if (c.pinned_n < need) {
        if (c.pinned) cudaFreeHost(c.pinned);
        c.pinned = nullptr;
        c.pinned_n = 0;
        ck(cudaHostAlloc(&c.pinned, need, cudaHostAllocDefault), "pinned staging");
        c.pinned_n = need;
    }
    double* hld = static_cast<double*>(c.pinned);
    double* hms = meansq_out ? hld + MK : nullptr;
    unsigned* hst = reinterpret_cast<unsigned*>(hld + MK * (meansq_out ? 2 : 1));

    struct Chunk {
        std::shared_ptr<Prepared> P;
        std::unique_ptr<WinPlan> plan;
        cudaEvent_t done = nullptr;
        bool copied = false;
    };
    std::vector<Chunk> ch(nc);
    const cudaStream_t st_main = c.st;
    struct Cleanup {
        Context& c;
        cudaStream_t st;
        std::vector<Chunk>& ch;
        ~Cleanup() {
            c.st = st;
            cudaStreamSynchronize(c.st_prep);
            cudaStreamSynchronize(st);
            for (Chunk& x : ch)
                if (x.done) cudaEventDestroy(x.done);
        }
    } cleanup{c, st_main, ch};
    auto copy_out = [&](size_t i) {
        const int64_t j0 = ws[cw[i]], L = ws[cw[i + 1]] - j0;
        if (hst[i]) fail(LDS_ERR_CUDA, "tensor-core pipeline wait timed out (code %u)", hst[i]);
        std::memcpy(ldscore + j0 * K, hld + j0 * K, sizeof(double) * (size_t)(L * K));
        if (meansq_out)
            std::memcpy(meansq_out + j0 * K, hms + j0 * K, sizeof(double) * (size_t)(L * K));
        if (inv_out) std::memcpy(inv_out + j0, ch[i].plan->inv.data(), sizeof(double) * (size_t)L);
        ch[i].copied = true;
    };
    for (size_t i = 0; i < nc; ++i) {
        const int64_t wa = cw[i], wb = cw[i + 1], j0 = ws[wa], L = ws[wb] - j0;
        std::vector<int64_t> lws((size_t)(wb - wa + 1));
        for (int64_t w = wa; w <= wb; ++w) lws[(size_t)(w - wa)] = ws[w] - j0;
        c.st = c.st_prep;
        {
            // Chunk-owned memory from the pool, in st_prep's order; the host
            // synchronizes st_prep before the library stream touches it.
            PoolScope scope(c.pool, c.st_prep);
            ch[i].P = prepare(c, bed_rows + j0 * row_bytes, row_bytes, n_total, L, row_sel, n_sel,
                              impute, iseed, ddof, "stream", nullptr, j0);
            ch[i].plan = win_plan_create(c, ch[i].P, annot + j0 * K, K, lws.data(), wb - wa,
                                         nvecs, step, vtile, seed, dist, eps, as_float, 0,
                                         chunk_gb, wa);
            ch[i].plan->p1_spc = std::max(0, p1_spc);
            ch[i].plan->ld_d.as<double>((size_t)(L * K));
            ch[i].plan->ms_d.as<double>((size_t)(L * K));
            ck(cudaStreamSynchronize(c.st_prep), "chunk set-up");
        }
        c.st = st_main;
        win_execute(c, *ch[i].plan);
        win_results_async(c, *ch[i].plan, hld + j0 * K, hms ? hms + j0 * K : nullptr, hst + i);
        ck(cudaEventCreateWithFlags(&ch[i].done, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ch[i].done, c.st), "event");
        if (i == 0) c.timings[0] = ms_since(t_start);
        // Copy out the chunks that have finished while later ones still run.
        for (size_t q = 0; q < i; ++q)
            if (!ch[q].copied && cudaEventQuery(ch[q].done) == cudaSuccess) copy_out(q);
        (void)cudaGetLastError();  // cudaEventQuery's cudaErrorNotReady is not an error
    }
    c.timings[1] = ms_since(t_start);
    for (size_t i = 0; i < nc; ++i) {
        if (ch[i].copied) continue;
        ck(cudaEventSynchronize(ch[i].done), "chunk results");
        copy_out(i);
    }
    c.timings[2] = ms_since(t_start);
    for (Chunk& x : ch) {
        x.plan.reset();
        x.P.reset();
    }
    c.timings[3] = ms_since(t_start);
}

// Control-variate outputs of a windowed plan; call before its first execute.
void win_set_cv(Context& c, WinPlan& pl, const double* annot, int split, int D) {
    if (pl.graph) fail(LDS_ERR_ARG, "set the control-variate outputs before the first execute");
    if (D != 0 && D != 4 && D != 8 && D != 15) fail(LDS_ERR_ARG, "band width D must be 0, 4, 8 or 15");
    const int64_t M = pl.P->g.M, K = pl.K;
    pl.split = split ? 1 : 0;
    pl.cv_D = D;
    const size_t MK = (size_t)(M * K), nout = MK * (size_t)pl.ntiles_out();
    pl.accum.as<double>(nout);
    if (D > 0) {
        h2d(pl.annot_d.as<double>(MK), annot, MK, c.st);
        std::vector<double> ls((size_t)M);
        d2h(ls.data(), static_cast<double*>(pl.lscale.p), (size_t)M, c.st);
        ck(cudaStreamSynchronize(c.st), "cv setup");
        for (double& v : ls) v = std::sqrt(v);
        h2d(pl.sqrt_ls.as<double>((size_t)M), ls.data(), (size_t)M, c.st);
        int32_t* cnt = pl.band_cnt.as<int32_t>((size_t)(M * (D + 1) * 4));
        double* xx = pl.xx.as<double>((size_t)(M * (D + 1)));
        launch_nn_band(pl.P->g, D, cnt, c.st);
        launch_nn_band_finish(M, D, cnt, static_cast<double*>(pl.P->d_mean.p),
                              static_cast<double*>(pl.P->d_sdinv.p), xx, c.st);
        pl.cvC.as<double>(nout);
        pl.cvMu.as<double>(MK);
        for (auto& e : pl.cv_ev)
            if (!e) ck(cudaEventCreate(&e), "event");
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(c.st), "cv setup");
    }
}

// Row-major phase 1 (phase1_compute_Xz_bed_chunk_rowmajor_impl,
// gwldcore.cpp:1925-2130): Xz2d (N x K*v, row-major) += the block's
// contribution; bins without members are left as they are.
template <typename T>
void phase1_bed_rowmajor_impl(const char* bed_prefix, const char* fam_path, int blk_start,
                              int blk_end, const int64_t* row_sel, int64_t n_row_sel, int ddof,
                              const T* annot, int64_t annot_rows, int64_t K, const T* inv_right,
                              int v_start, int v_count, int rand_dist, int has_seed, uint64_t seed,
                              T* Xz, int64_t xz_rows, int64_t xz_cols, int impute, int has_iseed,
                              uint64_t iseed, T* inv_out, double resvar_eps, const T* Cm,
                              const T* Rm, int64_t p, const T* gram) {
    if (xz_cols != K * v_count) fail(LDS_ERR_ARG, "Xz2d_chunk shape must be (N, B*v_count)");
    std::vector<T> tmp((size_t)(xz_rows * xz_cols), T(0));
    phase1_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof, annot,
                       annot_rows, K, inv_right, v_start, v_count, rand_dist, has_seed, seed,
                       tmp.data(), xz_rows, xz_cols, nullptr, impute, has_iseed, iseed, inv_out,
                       resvar_eps, Cm, Rm, p, gram);
    for (int64_t n = 0; n < xz_rows; ++n)
        for (int64_t q = 0; q < xz_cols; ++q) Xz[n * xz_cols + q] += tmp[(size_t)(q * xz_rows + n)];
}

// C, R (N x p and p x N, column-major) projection of a device panel X (N x Q,
// column-major FP64): X <- X - C (R X) (project_panel_inplace,
// gwldcore.cpp:1119-1132).
template <typename T>
void project_device(Context& c, double* X, int64_t N, int64_t Q, const T* Cm, const T* Rm,
                    int64_t p) {
    if (p <= 0 || N <= 0 || Q <= 0) return;
    std::vector<double> Cd((size_t)(N * p)), Rt((size_t)(N * p));
    for (int64_t a = 0; a < p; ++a)
        for (int64_t i = 0; i < N; ++i) {
            Cd[(size_t)(a * N + i)] = (double)Cm[a * N + i];
            Rt[(size_t)(a * N + i)] = (double)Rm[i * p + a];
        }
    DevBuf dC, dR, dcoef;
    double* c_ = dC.as<double>(Cd.size());
    double* r_ = dR.as<double>(Rt.size());
    h2d(c_, Cd.data(), Cd.size(), c.st);
    h2d(r_, Rt.data(), Rt.size(), c.st);
    const int mb = col_dots_max_basis();
    const int64_t nch = (p + mb - 1) / mb;
    double* coef = dcoef.as<double>((size_t)(Q * mb * nch));
    // all coefficients from the unprojected panel first, then the update
    for (int64_t ch = 0; ch < nch; ++ch) {
        const int nb = (int)std::min<int64_t>(mb, p - ch * mb);
        launch_col_dots(X, N, N, Q, r_ + ch * mb * N, N, nb, 0, coef + ch * Q * mb, c.st);
    }
    for (int64_t ch = 0; ch < nch; ++ch) {
        const int nb = (int)std::min<int64_t>(mb, p - ch * mb);
        launch_sub_lowrank(X, N, N, Q, c_ + ch * mb * N, N, nb, coef + ch * Q * mb, 0, 1.0, c.st);
    }
    ck(cudaGetLastError(), "launch");
    ck(cudaStreamSynchronize(c.st), "projection");
}

template <typename T>
void col_sums_rowmajor_impl(const T* X, int64_t N, int64_t Q, double* out) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (N <= 0 || Q <= 0) {
        for (int64_t q = 0; q < Q; ++q) out[q] = 0.0;
        return;
    }
    DevBuf dx, ds;
    T* x = dx.as<T>((size_t)(N * Q));
    h2d(x, X, (size_t)(N * Q), c.st);
    double* s = ds.as<double>((size_t)Q);
    launch_col_sums_rowmajor<T>(x, N, Q, s, c.st);
    ck(cudaGetLastError(), "launch");
    d2h(out, s, (size_t)Q, c.st);
    ck(cudaStreamSynchronize(c.st), "col sums");
}

template <typename T>
void project_rowmajor_impl(T* X, int64_t N, int64_t Q, const T* Cm, const T* Rm, int64_t p,
                           double* sums) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (N <= 0 || Q <= 0) {
        for (int64_t q = 0; q < Q; ++q) sums[q] = 0.0;
        return;
    }
    DevBuf dx, dcol, ds;
    T* x = dx.as<T>((size_t)(N * Q));
    h2d(x, X, (size_t)(N * Q), c.st);
    if (p > 0 && Cm && Rm) {
        double* col = dcol.as<double>((size_t)(N * Q));
        launch_rowmajor_to_colmajor<T>(x, N, Q, col, c.st);
        project_device<T>(c, col, N, Q, Cm, Rm, p);
        launch_colmajor_to_rowmajor<T>(col, N, Q, x, c.st);
        d2h(X, x, (size_t)(N * Q), c.st);
    }
    double* s = ds.as<double>((size_t)Q);
    launch_col_sums_rowmajor<T>(x, N, Q, s, c.st);
    ck(cudaGetLastError(), "launch");
    d2h(sums, s, (size_t)Q, c.st);
    ck(cudaStreamSynchronize(c.st), "projection");
}

template <typename T>
void project_colmajor_impl(T* X, int64_t N, int64_t Q, const T* Cm, const T* Rm, int64_t p) {
    if (N <= 0 || Q <= 0 || p <= 0 || !Cm || !Rm) return;
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    DevBuf dx, dcol;
    T* x = dx.as<T>((size_t)(N * Q));
    h2d(x, X, (size_t)(N * Q), c.st);
    double* col = dcol.as<double>((size_t)(N * Q));
    launch_convert<T>(x, N * Q, col, c.st);
    project_device<T>(c, col, N, Q, Cm, Rm, p);
    launch_convert_back<T>(col, N * Q, x, c.st);
    ck(cudaGetLastError(), "launch");
    d2h(X, x, (size_t)(N * Q), c.st);
    ck(cudaStreamSynchronize(c.st), "projection");
}

template <typename T>
int64_t standardize_dosage_impl(T* G, int64_t N, int64_t L, int ddof, double missing) {
    if (N <= 0) fail(LDS_ERR_ARG, "Dosage matrix must have at least one sample");
    if (L < 0) fail(LDS_ERR_ARG, "Invalid dosage matrix column count");
    if (L == 0) return 0;
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    DevBuf dg, dc;
    T* g = dg.as<T>((size_t)(N * L));
    h2d(g, G, (size_t)(N * L), c.st);
    unsigned long long* cnt = dc.as<unsigned long long>(2);
    ck(cudaMemsetAsync(cnt, 0, 16, c.st), "memset");
    launch_standardize_dosage<T>(g, N, L, ddof, missing, cnt, c.st);
    ck(cudaGetLastError(), "launch");
    unsigned long long hc[2] = {0, 0};
    d2h(G, g, (size_t)(N * L), c.st);
    d2h(hc, cnt, 2, c.st);
    ck(cudaStreamSynchronize(c.st), "standardize");
    if (hc[1]) fail(LDS_ERR_ARG, "Dosage matrix contains nonfinite or out-of-range nonmissing values");
    return (int64_t)hc[0];
}

// ---------------------------------------------------------------------------
// SUMMIT-GxE multi-environment products (MultiEnvironmentKernel,
// gxeldcore.cpp:10281-12557) on a resident genotype image.  The image's
// standardization (mean imputation, its ddof) is the genotype block the
// reference's driver passes (GenomewideEnvLDScore._read_genotype_block).
// ---------------------------------------------------------------------------
struct GxeCtx {
    // The resident image whose blocks the products read, or null for a
    // context that takes the reference's dense standardized genotype blocks.
    std::shared_ptr<Prepared> P;
    int64_t N = 0, N_pad = 0, E = 0, r = 0;
    int K = 0;
    std::vector<int32_t> ranks;
    DevBuf env, common, dirs_ones, ranks_d, ones_M;
    std::vector<DevBuf> basis0;          // per environment: N x rank fixed-effect basis
    // workspaces (grow-only)
    DevBuf probes, annot, sx, sw, panel, y, wq, wcs, rowind, sc, binoff, coef, coef2, denom;
    DevBuf sacc, acc4, guards, status, flag;
    DevBuf dgeno, dw, ones_L;            // dense-block path
    // Exact checks of the target's phase-2 products (lds_gxe_set_checks):
    // per-SNP checksums from the tensor-core epilogue (lhs) and from the
    // CUDA-core recomputation (rhs), and the last target call's result.
    int check = 0;
    DevBuf chk_lhs, chk_rhs, chk_u, chk_tiles;
    std::vector<unsigned long long> chk_hl, chk_hr;
    int64_t chk_j0 = 0, chk_rows = 0, chk_bad = 0, chk_first = -1;
};

struct GxePair {
    int64_t N = 0, C = 0, G = 0;
    DevBuf ypair;                        // N_pad x 2C FP64, rows N..N_pad zero
    int B = 0;                           // probe count the digits were made for
    DevBuf yq, ycs;
};

std::map<int64_t, std::unique_ptr<GxeCtx>>& gxe_table() {
    static std::map<int64_t, std::unique_ptr<GxeCtx>> t;
    return t;
}
std::map<int64_t, std::unique_ptr<GxePair>>& gxe_pair_table() {
    static std::map<int64_t, std::unique_ptr<GxePair>> t;
    return t;
}

// Device view of a caller array: the pointer itself, or a copy in `buf`.
template <typename T>
const T* dev_in(Context& c, DevBuf& buf, const T* p, size_t n, int device_ptrs) {
    if (device_ptrs || !p) return p;
    T* d = buf.as<T>(std::max<size_t>(n, 1));
    h2d(d, p, n, c.st);
    return d;
}

// source_block: target (N x T 2 K B, column-major) += the contribution of SNPs
// [j0, j1) (gxeldcore.cpp:11008-11240).
// With `dense` (N x (j1 - j0) column-major standardized genotypes, host or
// device memory as device_ptrs says) the block comes from the caller, as in
// the reference's binding; otherwise it is SNPs [j0, j1) of the image.
void gxe_source_impl(Context& c, GxeCtx& g, int64_t j0, int64_t j1, const double* probes, int64_t B,
                     const double* annot, int is_sqrt, const double* sx, const double* sw, int64_t T,
                     int env_start, double* target, int device_ptrs, const double* dense = nullptr) {
    const int64_t L = j1 - j0, N = g.N, Np = g.N_pad, K = g.K;
    if (!dense && !g.P) fail(LDS_ERR_ARG, "this kernel takes dense genotype blocks");
    if (B <= 0 || T <= 0 || env_start < 0 || env_start + T > g.E || L <= 0 || j0 < 0 ||
        (!dense && j1 > g.P->g.M))
        fail(LDS_ERR_ARG, "Multi-environment native source inputs have incompatible dimensions");
    const int64_t G = T * 2 * K, C = G * B;
    const double* dz = dev_in(c, g.probes, probes, (size_t)(L * B), device_ptrs);
    const double* da = dev_in(c, g.annot, annot, (size_t)(L * K), device_ptrs);
    const double* dsx = dev_in(c, g.sx, sx, (size_t)(L * T), device_ptrs);
    const double* dsw = dev_in(c, g.sw, sw, (size_t)(L * T), device_ptrs);
    unsigned* flag = g.flag.as<unsigned>(1);
    ck(cudaMemsetAsync(flag, 0, 4, c.st), "memset");
    launch_gxe_check(dz, L * B, dsx, dsw, L * T, da, is_sqrt ? 0 : L * K, flag, c.st);
    // Member lists need the annotation and scales on the host.
    std::vector<double> ha((size_t)(L * K)), hx((size_t)(L * T)), hw((size_t)(L * T));
    d2h(ha.data(), da, ha.size(), c.st);
    d2h(hx.data(), dsx, hx.size(), c.st);
    d2h(hw.data(), dsw, hw.size(), c.st);
    unsigned fv = 0;
    d2h(&fv, flag, 1, c.st);
    ck(cudaStreamSynchronize(c.st), "gxe inputs");
    if (fv) fail(LDS_ERR_ARG, "Multi-environment native source inputs contain invalid values");
    double* dtarget = device_ptrs ? target : g.panel.as<double>((size_t)(N * C));
    if (!device_ptrs) h2d(dtarget, target, (size_t)(N * C), c.st);
    if (dense) {
        // The caller's block is arbitrary FP64: weights[j, ((e 2 + h) K + k) B + b] =
        // sqrt(a_jk) s_h,e[j] z_jb (gxeldcore.cpp:11008-11240) and Y = X weights as
        // an FP64 product on the device.
        std::vector<double> hz((size_t)(L * B));
        d2h(hz.data(), dz, hz.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "gxe probes");
        std::vector<double> W((size_t)(L * C), 0.0);
        for (int64_t e = 0; e < T; ++e)
            for (int h = 0; h < 2; ++h) {
                const double* sh = (h == 0 ? hx.data() : hw.data()) + e * L;
                for (int64_t k = 0; k < K; ++k) {
                    const int64_t col0 = ((e * 2 + h) * K + k) * B;
                    for (int64_t j = 0; j < L; ++j) {
                        const double av = ha[(size_t)(k * L + j)];
                        const double sa = is_sqrt ? av : std::sqrt(std::max(0.0, av));
                        if (!(sa > 0.0)) continue;
                        const double f = sa * sh[j];
                        for (int64_t bq = 0; bq < B; ++bq)
                            W[(size_t)((col0 + bq) * L + j)] = f * hz[(size_t)(bq * L + j)];
                    }
                }
            }
        const double* dg = dev_in(c, g.dgeno, dense, (size_t)(N * L), device_ptrs);
        double* dW = g.dw.as<double>(W.size());
        h2d(dW, W.data(), W.size(), c.st);
        double* Y = g.y.as<double>((size_t)(Np * C));
        DGemmArgs ga;
        ga.M = N;
        ga.N = C;
        ga.K = L;
        ga.A = dg;
        ga.a_ms = 1;
        ga.a_ks = N;
        ga.B = dW;
        ga.b_ks = 1;
        ga.b_ns = L;
        ga.C = Y;
        ga.c_ms = 1;
        ga.c_ns = Np;
        launch_dgemm(ga, c.st);
        launch_gxe_source_finalize(Y, N, Np, C, (int)(K * B), static_cast<double*>(g.env.p), N,
                                   env_start, dtarget, N, c.st);
        ck(cudaGetLastError(), "launch");
        if (!device_ptrs) d2h(target, dtarget, (size_t)(N * C), c.st);
        ck(cudaStreamSynchronize(c.st), "gxe source");
        return;
    }
    const Prepared& P = *g.P;
    const int nc = umma::ncolp_for((int)B);
    // SNP chunks bound the weight-digit buffer (G x 2 x ncolp x chunk bytes).
    const int64_t cap = (int64_t)1 << 30;
    int64_t Lb = std::max<int64_t>(128, cap / std::max<int64_t>(1, G * 2 * nc) / 128 * 128);
    Lb = std::min(Lb, round_up(L, 128));
    double* Y = g.y.as<double>((size_t)(Np * C));
    for (int64_t a = 0; a < L; a += Lb) {
        const int64_t b = std::min(L, a + Lb), Lc = b - a;
        // Super-bin (e, h, k): members with sqrt(a_jk) > 0, scale sqrt(a_jk) s_h,e[j].
        std::vector<int64_t> off((size_t)G + 1, 0);
        std::vector<int32_t> ri;
        std::vector<double> scv;
        int64_t lmax = 128;
        for (int64_t e = 0; e < T; ++e)
            for (int h = 0; h < 2; ++h)
                for (int64_t k = 0; k < K; ++k) {
                    const int64_t gi = (e * 2 + h) * K + k;
                    off[(size_t)gi] = (int64_t)ri.size();
                    const double* s = (h == 0 ? hx.data() : hw.data()) + e * L;
                    for (int64_t j = a; j < b; ++j) {
                        const double av = ha[(size_t)(k * L + j)];
                        const double sa = is_sqrt ? av : std::sqrt(std::max(0.0, av));
                        if (!(sa > 0.0)) continue;
                        ri.push_back((int32_t)(j - a));
                        scv.push_back(sa * s[j]);
                    }
                    const int64_t n = (int64_t)ri.size() - off[(size_t)gi];
                    const int64_t np = round_up(n, 128);
                    for (int64_t q = n; q < np; ++q) {
                        ri.push_back(0);
                        scv.push_back(0.0);
                    }
                    lmax = std::max(lmax, np);
                }
        off[(size_t)G] = (int64_t)ri.size();
        const size_t nm = std::max<size_t>(ri.size(), 1);
        h2d(g.rowind.as<int32_t>(nm), ri.data(), ri.size(), c.st);
        h2d(g.sc.as<double>(nm), scv.data(), scv.size(), c.st);
        h2d(g.binoff.as<int64_t>(off.size()), off.data(), off.size(), c.st);
        const size_t wbytes = (size_t)(G * 2 * nc) * (size_t)lmax;
        int8_t* wq = g.wq.as<int8_t>(wbytes);
        ck(cudaMemsetAsync(wq, 0, wbytes, c.st), "memset weights");
        umma::P1UWeights uw;
        uw.K = (int)G;
        uw.V = (int)B;
        uw.ncolp = nc;
        uw.lmax = lmax;
        uw.rowind = static_cast<int32_t*>(g.rowind.p);
        uw.sc = static_cast<double*>(g.sc.p);
        uw.bin_off = static_cast<int64_t*>(g.binoff.p);
        uw.wq = wq;
        uw.colscale = g.wcs.as<double>((size_t)(G * B));
        const double* mean = static_cast<const double*>(P.d_mean.p) + j0 + a;
        const double* sdinv = static_cast<const double*>(P.d_sdinv.p) + j0 + a;
        umma::launch_p1_weights4(uw, mean, sdinv, dz + a, L, c.st);
        const CUtensorMap tmW = make_map_2d(wq, (uint64_t)lmax, (uint64_t)(G * 2 * nc), (uint64_t)lmax,
                                            128, (uint32_t)std::min(256, nc),
                                            CU_TENSOR_MAP_SWIZZLE_128B);
        umma::P1UArgs pa;
        pa.K = (int)G;
        pa.V = (int)B;
        pa.ncolp = nc;
        pa.ngroups = (nc + 255) / 256;
        pa.box_rows = std::min(256, nc);
        pa.nbp = P.g.nbp;
        pa.N_pad = Np;
        pa.bin_off = uw.bin_off;
        pa.rowind = uw.rowind;
        pa.codes = P.g.codes + (j0 + a) * P.g.nbp;
        pa.colscale = uw.colscale;
        pa.Y = Y;
        pa.status = g.status.as<unsigned>(1);
        ck(cudaMemsetAsync(pa.status, 0, 4, c.st), "memset");
        umma::launch_p1_umma(tmW, pa, Np, c.st);
        launch_gxe_source_finalize(Y, N, Np, C, (int)(K * B), static_cast<double*>(g.env.p), N,
                                   env_start, dtarget, N, c.st);
        unsigned stv = 0;
        d2h(&stv, pa.status, 1, c.st);
        ck(cudaStreamSynchronize(c.st), "gxe source");
        if (stv) fail(LDS_ERR_CUDA, "GxE source tensor-core pipeline wait timed out (code %u)", stv);
        (void)Lc;
    }
    if (!device_ptrs) {
        d2h(target, dtarget, (size_t)(N * C), c.st);
        ck(cudaStreamSynchronize(c.st), "gxe source copy");
    }
}

// project_sources (gxeldcore.cpp:11583-11729); leakages[e] for the tile.
void gxe_project_impl(Context& c, GxeCtx& g, double* panel, int64_t cols, int cpe, int env_start,
                      int device_ptrs, double* leakages) {
    const int64_t N = g.N;
    if (cpe <= 0 || cols % (2 * (int64_t)cpe) != 0)
        fail(LDS_ERR_ARG, "Multi-environment native projection panel is mis-sized");
    const int64_t T = cols / (2 * (int64_t)cpe);
    if (T <= 0 || env_start < 0 || env_start + T > g.E)
        fail(LDS_ERR_ARG, "Multi-environment native projection tile is outside the environment axis");
    double* dp = device_ptrs ? panel : g.panel.as<double>((size_t)(N * cols));
    if (!device_ptrs) h2d(dp, panel, (size_t)(N * cols), c.st);
    const int mb = col_dots_max_basis();
    // P <- P - U (U^T P), basis in chunks of mb columns
    for (int64_t a0 = 0; a0 < g.r; a0 += mb) {
        const int nb = (int)std::min<int64_t>(mb, g.r - a0);
        double* coef = g.coef.as<double>((size_t)(cols * nb));
        const double* U = static_cast<const double*>(g.common.p) + a0 * N;
        launch_col_dots(dp, N, N, cols, U, N, nb, 0, coef, c.st);
        launch_sub_lowrank(dp, N, N, cols, U, N, nb, coef, 0, 1.0, c.st);
    }
    // direction and mean from the same values: basis [d_e, 1]
    const int64_t seg = 2 * (int64_t)cpe;
    double* coef2 = g.coef2.as<double>((size_t)(seg * 2));
    for (int64_t e = 0; e < T; ++e) {
        double* v = dp + e * seg * N;
        const double* D = static_cast<const double*>(g.dirs_ones.p) + (env_start + e) * 2 * N;
        launch_col_dots(v, N, N, seg, D, N, 2, 0, coef2, c.st);
        launch_sub_lowrank(v, N, N, seg, D, N, 2, coef2, 1, 1.0 / (double)N, c.st);
    }
    // leakage onto each environment's fixed-effect basis
    std::vector<double> den((size_t)seg), co;
    for (int64_t e = 0; e < T; ++e) {
        const int env = (int)(env_start + e);
        const int rank = g.ranks[(size_t)env];
        double* v = dp + e * seg * N;
        double* dd = g.denom.as<double>((size_t)seg);
        launch_col_dots(v, N, N, seg, nullptr, N, 1, 1, dd, c.st);
        std::vector<double> leaked((size_t)seg, 0.0);
        d2h(den.data(), dd, (size_t)seg, c.st);
        for (int a0 = 0; a0 < rank; a0 += mb) {
            const int nb = std::min(mb, rank - a0);
            double* coef = g.coef.as<double>((size_t)(seg * nb));
            const double* B0 = static_cast<const double*>(g.basis0[(size_t)env].p) + (int64_t)a0 * N;
            launch_col_dots(v, N, N, seg, B0, N, nb, 0, coef, c.st);
            co.resize((size_t)(seg * nb));
            d2h(co.data(), coef, co.size(), c.st);
            ck(cudaStreamSynchronize(c.st), "gxe leakage");
            for (int64_t q = 0; q < seg; ++q)
                for (int a = 0; a < nb; ++a) leaked[(size_t)q] += co[(size_t)(q * nb + a)] * co[(size_t)(q * nb + a)];
        }
        ck(cudaStreamSynchronize(c.st), "gxe leakage");
        double maximum = 0.0;
        for (int64_t q = 0; q < seg; ++q) {
            const double rel = den[(size_t)q] > 0.0 ? std::sqrt(leaked[(size_t)q] / den[(size_t)q])
                                                    : std::numeric_limits<double>::infinity();
            if (!std::isfinite(rel)) fail(LDS_ERR_ARG, "Multi-environment native source leakage is non-finite");
            maximum = std::max(maximum, rel);
        }
        if (maximum > 1.0e-9)
            fail(LDS_ERR_ARG, "Multi-environment native source projection has excessive leakage");
        if (leakages) leakages[e] = maximum;
    }
    if (!device_ptrs) d2h(panel, dp, (size_t)(N * cols), c.st);
    ck(cudaStreamSynchronize(c.st), "gxe project");
}

// [right, w o right] sealed on the device (prepare_protected_row_weighted_pair,
// gxeldcore.cpp:9808); column c uses weight column c / (C / G).
std::unique_ptr<GxePair> gxe_pair_impl(Context& c, const GxeCtx& g, const double* right, int64_t N,
                                       int64_t C, const double* w, int64_t G, int device_ptrs) {
    if (N != g.N || C <= 0 || G <= 0 || C % G != 0)
        fail(LDS_ERR_ARG, "Protected GxE right-pair inputs have incompatible dimensions");
    auto pr = std::make_unique<GxePair>();
    pr->N = N;
    pr->C = C;
    pr->G = G;
    DevBuf tr, tw;
    const double* dr = dev_in(c, tr, right, (size_t)(N * C), device_ptrs);
    const double* dw = dev_in(c, tw, w, (size_t)(N * G), device_ptrs);
    double* yp = pr->ypair.as<double>((size_t)(g.N_pad * 2 * C));
    launch_gxe_pair(dr, N, N, g.N_pad, C, C / G, dw, N, 0, yp, c.st);
    ck(cudaGetLastError(), "launch");
    ck(cudaStreamSynchronize(c.st), "gxe pair");
    return pr;
}

// target_score_block (gxeldcore.cpp:11731-11936).
// SNPs whose G or O checksum pair differs (host comparison); the first one in
// *first (-1 if none).
static int64_t count_check_mismatches(const unsigned long long* lhs, const unsigned long long* rhs,
                                      int64_t n_snps, int64_t* first) {
    int64_t bad = 0, f = -1;
    for (int64_t j = 0; j < n_snps; ++j)
        if (lhs[2 * j] != rhs[2 * j] || lhs[2 * j + 1] != rhs[2 * j + 1]) {
            if (f < 0) f = j;
            ++bad;
        }
    if (first) *first = f;
    return bad;
}

void gxe_target_impl(Context& c, GxeCtx& g, int64_t j0, int64_t j1, GxePair& pr, const double* sx,
                     const double* sw, int64_t T, double* axx, double* axw, double* awx, double* aww,
                     int64_t block_start, int64_t total, int probe_count, int env_start,
                     int device_ptrs, const double* dense = nullptr) {
    const int64_t L = j1 - j0, N = g.N, Np = g.N_pad, K = g.K;
    if (!dense && !g.P) fail(LDS_ERR_ARG, "this kernel takes dense genotype blocks");
    if (block_start < 0 || total <= 0 || block_start + L > total || probe_count <= 0 || T <= 0 ||
        env_start < 0 || env_start + T > g.E || L <= 0 || j0 < 0 || (!dense && j1 > g.P->g.M))
        fail(LDS_ERR_ARG, "Multi-environment native target scale/block metadata is invalid");
    const int64_t B = probe_count, pair_cols = T * 2 * K * B;
    if (pr.N != N || pr.C != pair_cols)
        fail(LDS_ERR_ARG, "Multi-environment native target pair is incompatible with the tile");
    const int64_t Kp = 2 * T * 2 * K;
    const int nc = umma::ncolp_for((int)B);
    if (!dense && pr.B != (int)B) {
        int8_t* yq = pr.yq.as<int8_t>((size_t)(Kp * nc * Np));
        umma::launch_quantize_y4(static_cast<double*>(pr.ypair.p), N, Np, (int)Kp, (int)B, nc, yq,
                                 pr.ycs.as<double>((size_t)(Kp * B)), c.st);
        pr.B = (int)B;
    }
    const double* dsx = dev_in(c, g.sx, sx, (size_t)(L * T), device_ptrs);
    const double* dsw = dev_in(c, g.sw, sw, (size_t)(L * T), device_ptrs);
    unsigned* flag = g.flag.as<unsigned>(1);
    const bool checked = g.check && !dense;
    std::vector<int4> chk_tiles;  // rows of the check's CUDA-core pass (alive until the sync)
    ck(cudaMemsetAsync(flag, 0, 4, c.st), "memset");
    launch_gxe_check(dsx, 0, dsx, dsw, L * T, dsx, 0, flag, c.st);
    unsigned fv = 0;
    d2h(&fv, flag, 1, c.st);
    ck(cudaStreamSynchronize(c.st), "gxe scales");
    if (fv) fail(LDS_ERR_ARG, "Multi-environment native target scales contain invalid values");
    double* S = g.sacc.as<double>((size_t)(L * Kp));
    ck(cudaMemsetAsync(S, 0, sizeof(double) * (size_t)(L * Kp), c.st), "memset");
    unsigned* status = g.status.as<unsigned>(1);
    ck(cudaMemsetAsync(status, 0, 4, c.st), "memset");
    if (dense) {
        // Work = X^T [S, w o S] (L x 2C) as an FP64 product, then per (SNP,
        // group) the sum of squares over the group's B probes.
        const double* dg = dev_in(c, g.dgeno, dense, (size_t)(N * L), device_ptrs);
        double* Wk = g.dw.as<double>((size_t)(L * Kp * B));
        DGemmArgs ga;
        ga.M = L;
        ga.N = Kp * B;
        ga.K = N;
        ga.A = dg;
        ga.a_ms = N;
        ga.a_ks = 1;
        ga.B = static_cast<const double*>(pr.ypair.p);
        ga.b_ks = 1;
        ga.b_ns = Np;
        ga.C = Wk;
        ga.c_ms = 1;
        ga.c_ns = L;
        launch_dgemm(ga, c.st);
        if ((int64_t)(g.ones_L.n / sizeof(double)) < L) {
            std::vector<double> ones((size_t)L, 1.0);
            h2d(g.ones_L.as<double>((size_t)L), ones.data(), ones.size(), c.st);
        }
        unsigned long long* gd = g.guards.as<unsigned long long>(2);
        ck(cudaMemsetAsync(gd, 0, 16, c.st), "memset");
        launch_dense_p2_epilogue(Wk, L, (int)Kp, (int)B, static_cast<double*>(g.ones_L.p), S,
                                 nullptr, gd, std::numeric_limits<double>::infinity(), 0, c.st);
    } else {
    const Prepared& P = *g.P;
    // several groups per CTA in 256-column MMA groups (16 groups of 400
    // columns at B = 100: 50 MMA groups per SNP tile instead of 64)
    const int nb = umma::p2_bins_per_cta_grouped(nc, (int)Kp);
    umma::P2UArgs u;
    u.K = (int)Kp;
    u.V = (int)B;
    u.ncolp = nc;
    u.bins_per_cta = nb;
    u.ngroups = (nb * nc + 255) / 256;
    u.box_rows = std::min(256, nb * nc);
    u.nkt = (int)(Np / 128);
    u.M = P.g.M;
    u.j0 = j0;
    u.j1 = j1;
    u.out_row0 = j0;
    u.colscale = static_cast<double*>(pr.ycs.p);
    u.mean = static_cast<double*>(P.d_mean.p);
    u.sdinv = static_cast<double*>(P.d_sdinv.p);
    u.left_scale = static_cast<double*>(g.ones_M.p);
    u.accum = S;
    u.guard_counts = g.guards.as<unsigned long long>(2);
    u.extreme_warn = std::numeric_limits<double>::infinity();
    u.drop_extreme = 0;
    u.status = status;
    const CUtensorMap tmA = make_map_2d(P.g.codes, (uint64_t)P.g.nbp, (uint64_t)P.g.M_pad,
                                        (uint64_t)P.g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
    u.yq = static_cast<const int8_t*>(pr.yq.p);
    u.yq_cols = Kp * nc;
    unsigned long long *chk_lhs = nullptr, *chk_rhs = nullptr;
    if (checked) {
        // checksums indexed by SNP (the kernel writes 2 j, 2 j + 1)
        chk_lhs = g.chk_lhs.as<unsigned long long>((size_t)(2 * P.g.M));
        chk_rhs = g.chk_rhs.as<unsigned long long>((size_t)(2 * P.g.M));
        ck(cudaMemsetAsync(chk_lhs + 2 * j0, 0, sizeof(unsigned long long) * 2 * (size_t)L, c.st),
           "memset");
        ck(cudaMemsetAsync(chk_rhs + 2 * j0, 0, sizeof(unsigned long long) * 2 * (size_t)L, c.st),
           "memset");
        u.chk = chk_lhs;
        u.chk_v0 = 0;
    }
    umma::launch_p2_umma(tmA, u, c.st);
    if (checked) {
        // the same products on the CUDA cores: u(i) = sum_{k,v} h(k, v) y~_kv(i)
        // over the pair's digits, then sum_i g_ij u(i) and o_ij u(i) per SNP
        auto* ub = g.chk_u.as<unsigned long long>((size_t)Np);
        launch_check_u(static_cast<const int8_t*>(pr.yq.p), Kp * nc, nc, (int)Kp, (int)B, 0, 1, Np,
                       ub, c.st);
        for (int64_t j = j0; j < j1; j += 128)
            chk_tiles.push_back(make_int4((int)j, (int)j1, 0, 0));
        int4* dt = g.chk_tiles.as<int4>(chk_tiles.size());
        h2d(dt, chk_tiles.data(), chk_tiles.size(), c.st);
        launch_check_rhs(P.g.codes, P.g.nbp, dt, (int64_t)chk_tiles.size(), (int)Kp, ub, Np, chk_rhs,
                         c.st);
        g.chk_hl.resize(2 * (size_t)L);
        g.chk_hr.resize(2 * (size_t)L);
        d2h(g.chk_hl.data(), chk_lhs + 2 * j0, 2 * (size_t)L, c.st);
        d2h(g.chk_hr.data(), chk_rhs + 2 * j0, 2 * (size_t)L, c.st);
    }
    }
    const size_t nacc = (size_t)(g.E * total * K);
    double* A[4];
    if (device_ptrs) {
        A[0] = axx;
        A[1] = axw;
        A[2] = awx;
        A[3] = aww;
    } else {
        double* base = g.acc4.as<double>(4 * nacc);
        const double* hs[4] = {axx, axw, awx, aww};
        for (int q = 0; q < 4; ++q) {
            A[q] = base + (size_t)q * nacc;
            h2d(A[q], hs[q], nacc, c.st);
        }
    }
    launch_gxe_target_finalize(S, L, (int)Kp, (int)K, (int)T, dsx, dsw, L,
                               static_cast<int32_t*>(g.ranks_d.p), N, env_start, total, block_start,
                               A[0], A[1], A[2], A[3], c.st);
    ck(cudaGetLastError(), "launch");
    unsigned stv = 0;
    d2h(&stv, status, 1, c.st);
    if (!device_ptrs) {
        double* hs[4] = {axx, axw, awx, aww};
        for (int q = 0; q < 4; ++q) d2h(hs[q], A[q], nacc, c.st);
    }
    ck(cudaStreamSynchronize(c.st), "gxe target");
    if (stv) fail(LDS_ERR_CUDA, "GxE target tensor-core pipeline wait timed out (code %u)", stv);
    if (checked) {
        int64_t first = -1;
        g.chk_j0 = j0;
        g.chk_rows = L;
        g.chk_bad = count_check_mismatches(g.chk_hl.data(), g.chk_hr.data(), L, &first);
        g.chk_first = first < 0 ? -1 : j0 + first;
        if (g.chk_bad)
            fail(LDS_ERR_INTERNAL,
                 "GxE target product check failed: %lld SNPs disagree (first SNP %lld)",
                 (long long)g.chk_bad, (long long)g.chk_first);
    }
}

void gw_ldscore_impl(const uint8_t* bed_rows, int64_t row_bytes, int64_t n_total, int64_t M,
                     const int64_t* row_sel, int64_t n_sel, const double* annot, int64_t K,
                     int nvecs, int step, int vtile, uint64_t seed, int dist, int ddof,
                     int impute, uint64_t iseed, double eps, int as_float, double* ldscore,
                     double* meansq_out, double* inv_out, double* mc_agg, double* mc_snp) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    ensure_device(c);
    if (row_bytes < (n_total + 3) / 4) fail(LDS_ERR_ARG, "bed_row_bytes smaller than ceil(N/4)");
    if (impute != LDS_IMPUTE_MEAN && impute != LDS_IMPUTE_HWE)
        fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
    ck(cudaEventRecord(c.ev[0], c.st), "event");
    std::shared_ptr<Prepared> P(prepare(c, bed_rows, row_bytes, n_total, M, row_sel, n_sel, impute,
                                        iseed, ddof, "session"));
    ck(cudaEventRecord(c.ev[1], c.st), "event");
    auto pl = plan_create(c, P, annot, K, nvecs, step, vtile, seed, dist, eps, as_float,
                          (mc_agg || mc_snp) ? 1 : 0);
    plan_execute(c, *pl);
    plan_results(c, *pl, ldscore, meansq_out, inv_out, mc_agg, mc_snp);
    ck(cudaEventRecord(c.ev[5], c.st), "event");
    ck(cudaEventSynchronize(c.ev[5]), "sync");
    float up = 0.f, tot = 0.f;
    cudaEventElapsedTime(&up, c.ev[0], c.ev[1]);
    cudaEventElapsedTime(&tot, c.ev[0], c.ev[5]);
    c.timings[0] = up;
    c.timings[1] = pl->kernel_ms[0] + pl->kernel_ms[1];
    c.timings[2] = pl->kernel_ms[2] + pl->kernel_ms[3];
    c.timings[3] = tot;
}

}  // namespace

void set_last_error(const std::string& msg) { g_err = msg; }

double phase2_extreme_warn() { return extreme_warn_env(); }
int phase2_drop_extreme() { return drop_extreme_env(); }

// Setters registered by each file holding a copy of the bounded-wait limit.
// Registration runs during the library's static initialization (one thread);
// the list is read afterwards.
static std::vector<WaitLimitSetter>& wait_limit_setters() {
    static std::vector<WaitLimitSetter> v;
    return v;
}
void register_wait_limit_setter(WaitLimitSetter f) { wait_limit_setters().push_back(f); }
std::vector<CheckedErrSetter>& checked_err_setters() {
    static std::vector<CheckedErrSetter> v;
    return v;
}
void register_checked_err_setter(CheckedErrSetter f) { checked_err_setters().push_back(f); }
cudaError_t set_wait_limit_all(long long iters) {
    cudaError_t first = cudaSuccess;
    for (WaitLimitSetter f : wait_limit_setters()) {
        const cudaError_t e = f(iters);
        if (e != cudaSuccess && first == cudaSuccess) first = e;
    }
    return first;
}

}  // namespace lds

using namespace lds;

#define LDS_API extern "C" __attribute__((visibility("default")))

LDS_API const char* lds_last_error(void) { return g_err.c_str(); }

LDS_API const char* lds_version(void) {
    return "liblds 0.2 sm_100a (int8 digit-sliced exact products on tcgen05 tensor cores)";
}

LDS_API int lds_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

LDS_API int lds_set_slices(int s) {
    if (s < 3 || s > kMaxSlices) {
        g_err = "slices must be in [3, 6]";
        return LDS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx().mu);
    ctx().slices = s;
    return LDS_OK;
}

LDS_API int lds_get_slices(void) { return ctx().slices; }

LDS_API int lds_phase2_guard_counts(uint64_t* out2) {
    if (!out2) {
        g_err = "null output";
        return LDS_ERR_ARG;
    }
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    out2[0] = c.last_guards[0];
    out2[1] = c.last_guards[1];
    return LDS_OK;
}

// Bounded waits of the tensor-core kernels (see lds.h).
static std::atomic<long long> g_wait_limit{1LL << 25};

LDS_API int lds_set_wait_limit(long long iters) {
    if (iters < 1) {
        g_err = "wait limit must be >= 1";
        return LDS_ERR_ARG;
    }
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    return guarded([&] {
        ensure_device(c);
        // No library work may be in flight while the limit changes.
        ck(cudaStreamSynchronize(c.st), "wait limit");
        ck(set_wait_limit_all(iters), "wait limit");
        ck(cudaDeviceSynchronize(), "wait limit");
        g_wait_limit.store(iters);
    });
}

LDS_API long long lds_get_wait_limit(void) { return g_wait_limit.load(); }

LDS_API int lds_checked_build(void) {
#ifdef LDS_CHECKED
    return 1;
#else
    return 0;
#endif
}

LDS_API int lds_checked_errors(unsigned* code_out) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    return guarded([&] {
        if (!code_out) fail(LDS_ERR_ARG, "null output");
        *code_out = 0;
        if (!c.ready || !c.checked_err) return;
        ck(cudaStreamSynchronize(c.st), "sync");
        ck(cudaMemcpy(code_out, c.checked_err, sizeof(unsigned), cudaMemcpyDeviceToHost), "read");
        ck(cudaMemset(c.checked_err, 0, sizeof(unsigned)), "clear");
    });
}

LDS_API int lds_selftest_wait_timeout(unsigned* status_out) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    return guarded([&] {
        ensure_device(c);
        DevBuf d;
        unsigned* ds = d.as<unsigned>(1);
        ck(cudaMemsetAsync(ds, 0, sizeof(unsigned), c.st), "memset");
        launch_wait_timeout_probe(ds, c.st);
        ck(cudaGetLastError(), "launch");
        unsigned h = 0;
        d2h(&h, ds, 1, c.st);
        ck(cudaStreamSynchronize(c.st), "wait probe");
        if (status_out) *status_out = h;
    });
}

LDS_API uint64_t lds_kernel_launches(void) { return g_launches.load(); }

LDS_API void lds_clear_device_cache(void) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    c.cache.clear();
    for (auto& w : c.ws) w.reset();
    for (DevBuf* b : {&c.raw, &c.rows_dev, &c.hwe_q0, &c.hwe_q01, &c.hwe_sb, &c.counts_dev, &c.y,
                      &c.yq, &c.ycs, &c.wq, &c.wcs, &c.z, &c.rowind, &c.sc, &c.binoff, &c.wqoff,
                      &c.accum, &c.mc, &c.guards, &c.lscale, &c.xin, &c.units_dev, &c.colsum})
        b->release();
    if (c.pool) {
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(c.pool, 0);
    }
    if (c.pinned) cudaFreeHost(c.pinned);
    c.pinned = nullptr;
    c.pinned_n = 0;
}

#define P1_ARGS(T)                                                                              \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *annot_blk,                \
        int64_t annot_rows, int64_t K, const T *inv_right, int v_start, int v_count,            \
        int kmax_hint, int rand_dist, int has_seed, uint64_t seed, T *Xz2d_chunk,                \
        int64_t xz_rows, int64_t xz_cols, uint8_t *bin_init_mask, int impute_mode,              \
        int has_impute_seed, uint64_t impute_seed, T *inv_out, double resvar_eps, const T *C,   \
        const T *R, int64_t p, const T *resvar_gram, int project_right
#define P1_CALL(T)                                                                              \
    guarded([&] {                                                                               \
        (void)kmax_hint;                                                                        \
        phase1_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof,  \
                           annot_blk, annot_rows, K, inv_right, v_start, v_count, rand_dist,    \
                           has_seed, seed, Xz2d_chunk, xz_rows, xz_cols, bin_init_mask,         \
                           impute_mode, has_impute_seed, impute_seed, inv_out, resvar_eps, C,   \
                           R, p, resvar_gram, project_right);                                   \
    })
LDS_API int lds_phase1_compute_Xz_bed_chunk_f32(P1_ARGS(float)) { return P1_CALL(float); }
LDS_API int lds_phase1_compute_Xz_bed_chunk_f64(P1_ARGS(double)) { return P1_CALL(double); }

#define P2_ARGS(T)                                                                              \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,      \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,       \
        int64_t M_rows, int64_t K, int N_denom, int impute_mode, int has_impute_seed,           \
        uint64_t impute_seed, double *mc_aggregate_sumsq, double *mc_per_snp_sumsq, const T *C, \
        const T *R, int64_t p
#define P2_CALL(T)                                                                              \
    guarded([&] {                                                                               \
        phase2_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof,  \
                           inv_left, L, tile_nvecs, Xz2d, xz_rows, xz_cols, meansq_accum,       \
                           M_rows, K, N_denom, impute_mode, has_impute_seed, impute_seed,       \
                           mc_aggregate_sumsq, mc_per_snp_sumsq, C, R, p, 0);                   \
    })
LDS_API int lds_phase2_accum_XtXz_bed_f32(P2_ARGS(float)) { return P2_CALL(float); }
LDS_API int lds_phase2_accum_XtXz_bed_f64(P2_ARGS(double)) { return P2_CALL(double); }

#define P1R_ARGS(T)                                                                             \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *annot_blk,                \
        int64_t annot_rows, int64_t K, const T *inv_right, int v_start, int v_count,            \
        int kmax_hint, int rand_dist, int has_seed, uint64_t seed, T *Xz2d_chunk,                \
        int64_t xz_rows, int64_t xz_cols, int impute_mode, int has_impute_seed,                 \
        uint64_t impute_seed, T *inv_out, double resvar_eps, const T *C, const T *R, int64_t p, \
        const T *resvar_gram
#define P1R_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        (void)kmax_hint;                                                                        \
        phase1_bed_rowmajor_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel,          \
                                    n_row_sel, ddof, annot_blk, annot_rows, K, inv_right,       \
                                    v_start, v_count, rand_dist, has_seed, seed, Xz2d_chunk,    \
                                    xz_rows, xz_cols, impute_mode, has_impute_seed, impute_seed, \
                                    inv_out, resvar_eps, C, R, p, resvar_gram);                 \
    })
LDS_API int lds_phase1_compute_Xz_bed_chunk_rowmajor_f32(P1R_ARGS(float)) { return P1R_CALL(float); }
LDS_API int lds_phase1_compute_Xz_bed_chunk_rowmajor_f64(P1R_ARGS(double)) { return P1R_CALL(double); }

// Mailman phase 2 (gwldcore.cpp:2651-3119): HWE-completed genotypes, the same
// centered products on the tensor cores.
#define P2M_ARGS(T)                                                                             \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,      \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,       \
        int64_t M_rows, int64_t K, int N_denom, int has_impute_seed, uint64_t impute_seed,      \
        double *mc_aggregate_sumsq, double *mc_per_snp_sumsq, const T *C, const T *R, int64_t p
#define P2M_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        phase2_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof,  \
                           inv_left, L, tile_nvecs, Xz2d, xz_rows, xz_cols, meansq_accum,       \
                           M_rows, K, N_denom, LDS_IMPUTE_HWE, has_impute_seed, impute_seed,    \
                           mc_aggregate_sumsq, mc_per_snp_sumsq, C, R, p, 1);                   \
    })
LDS_API int lds_phase2_accum_XtXz_bed_mailman_f32(P2M_ARGS(float)) { return P2M_CALL(float); }
LDS_API int lds_phase2_accum_XtXz_bed_mailman_f64(P2M_ARGS(double)) { return P2M_CALL(double); }

// Row-major sketch with its column sums (gwldcore.cpp:2919-3119); the sums are
// recomputed exactly on the device, sum_Xz is checked for shape only.
#define P2MR_ARGS(T)                                                                            \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,      \
        int tile_nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum,       \
        int64_t M_rows, int64_t K, const double *sum_Xz, int64_t n_sum, int N_denom,            \
        int has_impute_seed, uint64_t impute_seed, double *mc_aggregate_sumsq,                  \
        double *mc_per_snp_sumsq
#define P2MR_CALL(T)                                                                            \
    guarded([&] {                                                                               \
        if (!sum_Xz || n_sum != xz_cols)                                                        \
            fail(LDS_ERR_ARG, "sum_Xz length must equal the Xz2d column count");                \
        std::vector<T> f((size_t)(xz_rows * xz_cols));                                          \
        for (int64_t n = 0; n < xz_rows; ++n)                                                   \
            for (int64_t q = 0; q < xz_cols; ++q)                                               \
                f[(size_t)(q * xz_rows + n)] = Xz2d[n * xz_cols + q];                          \
        phase2_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof,  \
                           inv_left, L, tile_nvecs, f.data(), xz_rows, xz_cols, meansq_accum,   \
                           M_rows, K, N_denom, LDS_IMPUTE_HWE, has_impute_seed, impute_seed,    \
                           mc_aggregate_sumsq, mc_per_snp_sumsq);                               \
    })
LDS_API int lds_phase2_accum_XtXz_bed_mailman_rowmajor_f32(P2MR_ARGS(float)) { return P2MR_CALL(float); }
LDS_API int lds_phase2_accum_XtXz_bed_mailman_rowmajor_f64(P2MR_ARGS(double)) { return P2MR_CALL(double); }

LDS_API int lds_compute_col_sums_rowmajor_f32(const float* X, int64_t N, int64_t Q, double* out) {
    return guarded([&] { col_sums_rowmajor_impl<float>(X, N, Q, out); });
}
LDS_API int lds_compute_col_sums_rowmajor_f64(const double* X, int64_t N, int64_t Q, double* out) {
    return guarded([&] { col_sums_rowmajor_impl<double>(X, N, Q, out); });
}
LDS_API int lds_project_rowmajor_inplace_and_col_sums_f32(float* X, int64_t N, int64_t Q,
                                                          const float* C, const float* R,
                                                          int64_t p, double* sums) {
    return guarded([&] { project_rowmajor_impl<float>(X, N, Q, C, R, p, sums); });
}
LDS_API int lds_project_rowmajor_inplace_and_col_sums_f64(double* X, int64_t N, int64_t Q,
                                                          const double* C, const double* R,
                                                          int64_t p, double* sums) {
    return guarded([&] { project_rowmajor_impl<double>(X, N, Q, C, R, p, sums); });
}
LDS_API int lds_project_colmajor_inplace_f32(float* X, int64_t N, int64_t Q, const float* C,
                                             const float* R, int64_t p) {
    return guarded([&] { project_colmajor_impl<float>(X, N, Q, C, R, p); });
}
LDS_API int lds_project_colmajor_inplace_f64(double* X, int64_t N, int64_t Q, const double* C,
                                             const double* R, int64_t p) {
    return guarded([&] { project_colmajor_impl<double>(X, N, Q, C, R, p); });
}
LDS_API int lds_standardize_dosage_inplace_f32(float* G, int64_t N, int64_t L, int ddof,
                                               double missing_value, int64_t* missing_out) {
    return guarded([&] {
        const int64_t mt = standardize_dosage_impl<float>(G, N, L, ddof, missing_value);
        if (missing_out) *missing_out = mt;
    });
}
LDS_API int lds_standardize_dosage_inplace_f64(double* G, int64_t N, int64_t L, int ddof,
                                               double missing_value, int64_t* missing_out) {
    return guarded([&] {
        const int64_t mt = standardize_dosage_impl<double>(G, N, L, ddof, missing_value);
        if (missing_out) *missing_out = mt;
    });
}

#define RV_ARGS(T)                                                                              \
    const char *bed_prefix, const char *fam_path, int nsnps, int step_size,                     \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, double eps, int impute_mode,       \
        int has_impute_seed, uint64_t impute_seed, T *inv_out, const T *C, const T *R,          \
        int64_t p, double *snp_var_out, int compute_mu22, const T *annot_all, int64_t annot_rows, \
        int64_t B, double *mu22_out
#define RV_CALL(T)                                                                              \
    guarded([&] {                                                                               \
        if (step_size <= 0)                                                                     \
            fail(LDS_ERR_ARG, "step_size must be > 0 in precompute_residual_variances_bed");     \
        if (compute_mu22 && !mu22_out) fail(LDS_ERR_ARG, "mu22_out is NULL");                   \
        resvar_impl<T>(bed_prefix, fam_path, nsnps, row_sel, n_row_sel, ddof, eps, impute_mode, \
                       has_impute_seed, impute_seed, inv_out, C, R, p, snp_var_out, annot_all,  \
                       annot_rows, B, compute_mu22 ? mu22_out : nullptr);                       \
    })
LDS_API int lds_precompute_residual_variances_bed_f32(RV_ARGS(float)) { return RV_CALL(float); }
LDS_API int lds_precompute_residual_variances_bed_f64(RV_ARGS(double)) { return RV_CALL(double); }

#define P1G_ARGS(T)                                                                             \
    const T *geno, int64_t N, int64_t L, int blk_start, const T *annot_blk, int64_t annot_rows,  \
        int64_t K, const T *inv_right, int v_start, int v_count, int kmax_hint, int rand_dist,  \
        int has_seed, uint64_t seed, T *Xz2d_chunk, int64_t xz_rows, int64_t xz_cols,            \
        uint8_t *bin_init_mask, const T *C, const T *R, int64_t p, const T *resvar_gram,         \
        T *inv_out, double resvar_eps
#define P1G_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        (void)kmax_hint;                                                                        \
        phase1_geno_impl<T>(geno, N, L, blk_start, annot_blk, annot_rows, K, inv_right, v_start, \
                            v_count, rand_dist, has_seed, seed, Xz2d_chunk, xz_rows, xz_cols,   \
                            bin_init_mask, inv_out, resvar_eps, C, R, p, resvar_gram);          \
    })
LDS_API int lds_phase1_compute_Xz_geno_chunk_f32(P1G_ARGS(float)) { return P1G_CALL(float); }
LDS_API int lds_phase1_compute_Xz_geno_chunk_f64(P1G_ARGS(double)) { return P1G_CALL(double); }

#define P2G_ARGS(T)                                                                             \
    T *geno, int64_t N, int64_t L, int blk_start, const T *inv_left, int64_t L_in, int tile_nvecs, \
        const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq_accum, int64_t M_rows,        \
        int64_t K, const T *C, const T *R, int64_t p, int N_denom, double *mc_aggregate_sumsq,   \
        double *mc_per_snp_sumsq
#define P2G_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        phase2_geno_impl<T>(geno, N, L, blk_start, inv_left, L_in, tile_nvecs, Xz2d, xz_rows,   \
                            xz_cols, meansq_accum, M_rows, K, C, R, p, N_denom,                 \
                            mc_aggregate_sumsq, mc_per_snp_sumsq);                              \
    })
LDS_API int lds_phase2_accum_XtXz_geno_f32(P2G_ARGS(float)) { return P2G_CALL(float); }
LDS_API int lds_phase2_accum_XtXz_geno_f64(P2G_ARGS(double)) { return P2G_CALL(double); }

// Legacy direct form (gwldcore.cpp:2132-2327): meansq += the guarded
// sum_c Work^2 inv^2 / (nvecs (N_denom - 1)^2); no Monte-Carlo sums.
#define P2L_ARGS(T)                                                                             \
    const char *bed_prefix, const char *fam_path, int blk_start, int blk_end,                   \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_left, int64_t L,      \
        int nvecs, const T *Xz2d, int64_t xz_rows, int64_t xz_cols, T *meansq, int64_t M_rows,  \
        int64_t K, const T *C, const T *R, int64_t p, int N_denom, int impute_mode,             \
        int has_impute_seed, uint64_t impute_seed
#define P2L_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        if (nvecs <= 0 || xz_cols % nvecs)                                                      \
            fail(LDS_ERR_ARG, "Xz2d col count must be multiple of nvecs");                       \
        phase2_bed_impl<T>(bed_prefix, fam_path, blk_start, blk_end, row_sel, n_row_sel, ddof,  \
                           inv_left, L, nvecs, Xz2d, xz_rows, xz_cols, meansq, M_rows, K,       \
                           N_denom, impute_mode, has_impute_seed, impute_seed, nullptr, nullptr, \
                           C, R, p, 0, 1.0 / (double)nvecs, "direct");                          \
    })
LDS_API int lds_phase2_compute_XtXz_bed_f32(P2L_ARGS(float)) { return P2L_CALL(float); }
LDS_API int lds_phase2_compute_XtXz_bed_f64(P2L_ARGS(double)) { return P2L_CALL(double); }

#define GRM_ARGS(T)                                                                             \
    const char *bed_prefix, const char *fam_path, int nsnps, int step_size,                     \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_all, int64_t n_inv,   \
        const T *panel_in, T *panel_out, int64_t rows, int64_t Q, const T *C, const T *R,       \
        int64_t p, int impute_mode, int has_impute_seed, uint64_t impute_seed
#define GRM_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        apply_grm_impl<T>(bed_prefix, fam_path, nsnps, step_size, row_sel, n_row_sel, ddof,     \
                          inv_all, n_inv, panel_in, panel_out, rows, Q, C, R, p, impute_mode,   \
                          has_impute_seed, impute_seed, "apply_grm_bed_panel");                 \
    })
LDS_API int lds_apply_grm_bed_panel_f32(GRM_ARGS(float)) { return GRM_CALL(float); }
LDS_API int lds_apply_grm_bed_panel_f64(GRM_ARGS(double)) { return GRM_CALL(double); }

// Mailman form (gwldcore.cpp:1256-1497): HWE-completed genotypes.
#define GRMM_ARGS(T)                                                                            \
    const char *bed_prefix, const char *fam_path, int nsnps, int step_size,                     \
        const int64_t *row_sel, int64_t n_row_sel, int ddof, const T *inv_all, int64_t n_inv,   \
        const T *panel_in, T *panel_out, int64_t rows, int64_t Q, const T *C, const T *R,       \
        int64_t p, int has_impute_seed, uint64_t impute_seed
#define GRMM_CALL(T)                                                                            \
    guarded([&] {                                                                               \
        apply_grm_impl<T>(bed_prefix, fam_path, nsnps, step_size, row_sel, n_row_sel, ddof,     \
                          inv_all, n_inv, panel_in, panel_out, rows, Q, C, R, p, LDS_IMPUTE_HWE, \
                          has_impute_seed, impute_seed, "apply_grm_bed_panel_mailman");         \
    })
LDS_API int lds_apply_grm_bed_panel_mailman_f32(GRMM_ARGS(float)) { return GRMM_CALL(float); }
LDS_API int lds_apply_grm_bed_panel_mailman_f64(GRMM_ARGS(double)) { return GRMM_CALL(double); }

#define BCB_ARGS(T)                                                                             \
    const double *meansq_raw, int64_t M, int64_t B, const double *mu22, const T *annot_all,     \
        int N, double d, double *R2, double *rho2, double *bias, double *delta
#define BCB_CALL(T)                                                                             \
    guarded([&] {                                                                               \
        block_corrections_impl<T>(meansq_raw, mu22, annot_all, M, B, N, d, R2, rho2, bias,      \
                                  delta);                                                       \
    })
LDS_API int lds_compute_block_corrections_binary_f32(BCB_ARGS(float)) { return BCB_CALL(float); }
LDS_API int lds_compute_block_corrections_binary_f64(BCB_ARGS(double)) { return BCB_CALL(double); }

LDS_API int lds_gw_ldscore(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total,
                           int64_t M, const int64_t* row_sel, int64_t n_row_sel,
                           const double* annot, int64_t K, int nvecs, int step_size, int vtile,
                           uint64_t seed, int rand_dist, int ddof, int impute_mode,
                           uint64_t impute_seed, double resvar_eps, int as_float, double* ldscore,
                           double* meansq_accum, double* inv_out, double* mc_aggregate_sumsq,
                           double* mc_per_snp_sumsq) {
    return guarded([&] {
        gw_ldscore_impl(bed_rows, bed_row_bytes, n_total, M, row_sel, n_row_sel, annot, K, nvecs,
                        step_size, vtile, seed, rand_dist, ddof, impute_mode, impute_seed,
                        resvar_eps, as_float, ldscore, meansq_accum, inv_out, mc_aggregate_sumsq,
                        mc_per_snp_sumsq);
    });
}

LDS_API int lds_gw_ldscore_bed(const char* bed_prefix, const char* fam_path,
                               const int64_t* row_sel, int64_t n_row_sel, const double* annot,
                               int64_t K, int nvecs, int step_size, int vtile, uint64_t seed,
                               int rand_dist, int ddof, int impute_mode, uint64_t impute_seed,
                               double resvar_eps, int as_float, double* ldscore,
                               double* meansq_accum, double* inv_out, double* mc_aggregate_sumsq,
                               double* mc_per_snp_sumsq) {
    return guarded([&] {
        const std::string bed = std::string(bed_prefix) + ".bed";
        const int64_t n_total = count_lines(fam_path);
        const int64_t M = count_lines(std::string(bed_prefix) + ".bim");
        MappedBed mb(bed);
        const int64_t nbytes = (n_total + 3) / 4;
        if ((size_t)(3 + M * nbytes) > mb.size) fail(LDS_ERR_IO, "BED file too small: %s", bed.c_str());
        gw_ldscore_impl(mb.base + 3, nbytes, n_total, M, row_sel, n_row_sel, annot, K, nvecs,
                        step_size, vtile, seed, rand_dist, ddof, impute_mode, impute_seed,
                        resvar_eps, as_float, ldscore, meansq_accum, inv_out, mc_aggregate_sumsq,
                        mc_per_snp_sumsq);
    });
}

LDS_API int lds_debug_xt_products(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n,
                                  int64_t L, const int8_t* y, int64_t Q, int64_t* out_g,
                                  int64_t* out_o) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (L <= 0 || Q <= 0 || n <= 0) fail(LDS_ERR_ARG, "invalid sizes");
        auto P = prepare(c, bed_rows, bed_row_bytes, n, L, nullptr, 0, LDS_IMPUTE_MEAN, 0, 1,
                         "debug");
        const int64_t Np = P->g.N_pad, Vp = round_up(Q, kColTile);
        std::vector<int8_t> yq((size_t)(Vp * Np), 0);
        for (int64_t q = 0; q < Q; ++q) std::memcpy(&yq[(size_t)(q * Np)], y + q * n, (size_t)n);
        int8_t* d_yq = c.yq.as<int8_t>(yq.size());
        h2d(d_yq, yq.data(), yq.size(), c.st);
        DevBuf rg, ro;
        long long* dg = rg.as<long long>((size_t)(L * Q));
        long long* dO = ro.as<long long>((size_t)(L * Q));
        P2Args a;
        a.K = 1;
        a.V = (int)Q;
        a.Vp = (int)Vp;
        a.S = 1;
        a.j0 = 0;
        a.j1 = L;
        a.out_row0 = 0;
        a.Yq = d_yq;
        a.raw_g = dg;
        a.raw_o = dO;
        launch_p2(P->g, a, c.st);
        ck(cudaGetLastError(), "launch");
        d2h(reinterpret_cast<long long*>(out_g), dg, (size_t)(L * Q), c.st);
        d2h(reinterpret_cast<long long*>(out_o), dO, (size_t)(L * Q), c.st);
        ck(cudaStreamSynchronize(c.st), "debug products");
    });
}

LDS_API int lds_set_stream(void* stream) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        static cudaStream_t own = c.st;
        c.st = stream ? static_cast<cudaStream_t>(stream) : own;
    });
}

LDS_API int lds_geno_create(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total,
                            int64_t M, const int64_t* row_sel, int64_t n_row_sel, int impute_mode,
                            uint64_t impute_seed, int ddof, int64_t* handle_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (bed_row_bytes < (n_total + 3) / 4) fail(LDS_ERR_ARG, "bed_row_bytes smaller than ceil(N/4)");
        if (impute_mode != LDS_IMPUTE_MEAN && impute_mode != LDS_IMPUTE_HWE)
            fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
        std::shared_ptr<Prepared> P(prepare(c, bed_rows, bed_row_bytes, n_total, M, row_sel,
                                            n_row_sel, impute_mode, impute_seed, ddof, "handle"));
        const int64_t h = next_handle();
        geno_table()[h] = P;
        *handle_out = h;
    });
}

LDS_API int lds_geno_create_synthetic(int64_t n_total, int64_t M, uint64_t seed,
                                      const int64_t* t0, const int64_t* t1, int missing,
                                      int impute_mode, uint64_t impute_seed, int ddof,
                                      int64_t* handle_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (n_total <= 0 || M <= 0) fail(LDS_ERR_ARG, "invalid sizes");
        if (impute_mode != LDS_IMPUTE_MEAN && impute_mode != LDS_IMPUTE_HWE)
            fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
        const SynthSpec spec{seed, t0, t1, missing};
        std::shared_ptr<Prepared> P(prepare(c, nullptr, (n_total + 3) / 4, n_total, M, nullptr, 0,
                                            impute_mode, impute_seed, ddof, "synthetic", &spec));
        const int64_t h = next_handle();
        geno_table()[h] = P;
        *handle_out = h;
    });
}

LDS_API int lds_geno_destroy(int64_t handle) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        geno_table().erase(handle);
    });
}

LDS_API int lds_geno_stats(int64_t geno, double* mean_out, double* sdinv_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        const Prepared& P = *it->second;
        if (mean_out) std::memcpy(mean_out, P.mean.data(), sizeof(double) * P.mean.size());
        if (sdinv_out) std::memcpy(sdinv_out, P.sdinv.data(), sizeof(double) * P.sdinv.size());
    });
}

// ---------------------------------------------------------------------------
// Exact windowed LD scores (compute_windowed_ld_chr_impl, winldcore.cpp:783-931)
// ---------------------------------------------------------------------------
// Per SNP the centering mean and rs = 1/sqrt(c_jj), c_jj = sum_obs (g - mu)^2,
// from the exact code counts (after HWE completion when that mode is used).
// The numerator Q nobs - S^2 is an exact integer.
void pearson_stats(const Prepared& P, int64_t j0, int64_t j1, std::vector<double>& mu,
                   std::vector<double>& rs) {
    mu.assign((size_t)P.g.M, 0.0);
    rs.assign((size_t)P.g.M, 0.0);
    for (int64_t j = j0; j < j1; ++j) {
        const SnpCounts& k = P.counts[(size_t)j];
        const long long nobs = (long long)k.n[0] + k.n[1] + k.n[2];
        const long long S = (long long)k.n[1] + 2LL * k.n[2];
        const long long Q = (long long)k.n[1] + 4LL * k.n[2];
        if (nobs <= 0) continue;
        mu[(size_t)j] = (double)S / (double)nobs;
        const long long num = Q * nobs - S * S;
        if (num > 0) rs[(size_t)j] = 1.0 / std::sqrt((double)num / (double)nobs);
    }
}

// LD[j, b] = sum_{i in [lo_j, hi_j)} f(r_ij) annot[i, b] for j in [row0, row1);
// lo/hi are SNP indices (clamped to the range), annot row-major (j - row0) K + b,
// f = r^2 (corr_dim <= 0) or the unbiased r^2 - (1 - r^2)/(corr_dim - 1).
// Output out[(j - row0) ld_row + b ld_col] (host).
void window_ld_impl(Context& c, const Prepared& P, int64_t row0, int64_t row1, const int64_t* lo,
                    const int64_t* hi, const double* annot, int64_t K, double corr_dim,
                    double* out, int64_t ld_row, int64_t ld_col) {
    const int64_t m = row1 - row0;
    if (row0 < 0 || row1 > P.g.M || m <= 0) fail(LDS_ERR_ARG, "SNP range outside the genotype image");
    if (K <= 0) fail(LDS_ERR_ARG, "annot_chr must have at least one column");
    if (corr_dim > 0.0 && corr_dim <= 1.0)
        fail(LDS_ERR_ARG, "Too few residual dimensions for unbiased windowed r^2 correction");
    std::vector<double> mu, rs;
    pearson_stats(P, row0, row1, mu, rs);
    std::vector<int32_t> lo32((size_t)m), hi32((size_t)m);
    for (int64_t r = 0; r < m; ++r) {
        lo32[(size_t)r] = (int32_t)std::min(row1, std::max(row0, lo[r]));
        hi32[(size_t)r] = (int32_t)std::min(row1, std::max(row0, hi[r]));
    }
    constexpr int64_t TB = 128;
    const int64_t nT = (m + TB - 1) / TB;
    // Partner tiles of each row tile, on the same 128-grid from row0.
    std::vector<std::pair<int64_t, int64_t>> span((size_t)nT, {0, 0});
    int64_t pairs = 0;
    for (int64_t T = 0; T < nT; ++T) {
        const int64_t a0 = T * TB, a1 = std::min(m, a0 + TB);
        int64_t lmin = row1, hmax = row0;
        for (int64_t r = a0; r < a1; ++r) {
            if (hi32[(size_t)r] <= lo32[(size_t)r]) continue;
            lmin = std::min<int64_t>(lmin, lo32[(size_t)r]);
            hmax = std::max<int64_t>(hmax, hi32[(size_t)r]);
        }
        if (hmax > lmin) {
            span[(size_t)T] = {(lmin - row0) / TB, (hmax - 1 - row0) / TB + 1};
            pairs += span[(size_t)T].second - span[(size_t)T].first;
        }
    }
    const int64_t per_cta = std::max<int64_t>(1, std::min<int64_t>(8, pairs / (148 * 4)));
    std::vector<int4> items;
    std::vector<int32_t> slot_beg((size_t)nT + 1, 0);
    for (int64_t T = 0; T < nT; ++T) {
        for (int64_t u = span[(size_t)T].first; u < span[(size_t)T].second; u += per_cta)
            items.push_back(make_int4((int)(row0 + T * TB), (int)(row0 + u * TB),
                                      (int)std::min(per_cta, span[(size_t)T].second - u),
                                      (int)items.size()));
        slot_beg[(size_t)T + 1] = (int32_t)items.size();
    }
    DevBuf d_items, d_beg, d_lo, d_hi, d_mu, d_rs, d_annot, d_part, d_out, d_st;
    const size_t nit = std::max<size_t>(items.size(), 1);
    int4* di = d_items.as<int4>(nit);
    h2d(di, items.data(), items.size(), c.st);
    int32_t* db = d_beg.as<int32_t>(slot_beg.size());
    h2d(db, slot_beg.data(), slot_beg.size(), c.st);
    int32_t* dlo = d_lo.as<int32_t>((size_t)m);
    int32_t* dhi = d_hi.as<int32_t>((size_t)m);
    h2d(dlo, lo32.data(), (size_t)m, c.st);
    h2d(dhi, hi32.data(), (size_t)m, c.st);
    double* dmu = d_mu.as<double>(mu.size());
    double* drs = d_rs.as<double>(rs.size());
    h2d(dmu, mu.data(), mu.size(), c.st);
    h2d(drs, rs.data(), rs.size(), c.st);
    double* dan = d_annot.as<double>((size_t)(m * K));
    h2d(dan, annot, (size_t)(m * K), c.st);
    const size_t npart = nit * (size_t)TB * (size_t)K;
    double* dpart = d_part.as<double>(npart);
    ck(cudaMemsetAsync(dpart, 0, npart * sizeof(double), c.st), "memset partial");
    double* dout = d_out.as<double>((size_t)(m * K));
    unsigned* dst = d_st.as<unsigned>(1);
    ck(cudaMemsetAsync(dst, 0, 4, c.st), "memset");
    GramArgs ga;
    ga.nkt = (int)(P.g.N_pad / 128);
    ga.K = (int)K;
    ga.row0 = row0;
    ga.row1 = row1;
    ga.items = di;
    ga.lo = dlo;
    ga.hi = dhi;
    ga.mean = dmu;
    ga.rs = drs;
    ga.annot = dan;
    ga.corr_den = corr_dim > 0.0 ? 1.0 / (corr_dim - 1.0) : 0.0;
    ga.partial = dpart;
    ga.status = dst;
    const CUtensorMap tmC = make_map_2d(P.g.codes, (uint64_t)P.g.nbp, (uint64_t)P.g.M_pad,
                                        (uint64_t)P.g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
    ck(cudaEventRecord(c.ev[0], c.st), "event");
    launch_gram_ld(tmC, ga, (int)items.size(), c.st);
    ck(cudaEventRecord(c.ev[2], c.st), "event");
    launch_gram_reduce(dpart, db, row0, row1, (int)K, dout, K, 1, c.st);
    ck(cudaEventRecord(c.ev[1], c.st), "event");
    ck(cudaGetLastError(), "launch");
    std::vector<double> h((size_t)(m * K));
    d2h(h.data(), dout, h.size(), c.st);
    unsigned stv = 0;
    d2h(&stv, dst, 1, c.st);
    ck(cudaStreamSynchronize(c.st), "windowed LD");
    if (stv) fail(LDS_ERR_CUDA, "windowed LD tensor-core pipeline wait timed out (code %u)", stv);
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]), "elapsed");
    c.timings[0] = ms;
    ck(cudaEventElapsedTime(&ms, c.ev[0], c.ev[2]), "elapsed");
    c.timings[1] = ms;  // Gram kernel alone
    for (int64_t r = 0; r < m; ++r)
        for (int64_t b = 0; b < K; ++b) out[r * ld_row + b * ld_col] = h[(size_t)(r * K + b)];
}

LDS_API int lds_geno_window_ld(int64_t geno, int64_t row0, int64_t row1, const int64_t* lo,
                               const int64_t* hi, const double* annot, int64_t K,
                               double corr_dim, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        if (!lo || !hi || !annot || !out) fail(LDS_ERR_ARG, "null argument");
        window_ld_impl(c, *it->second, row0, row1, lo, hi, annot, K, corr_dim, out, K, 1);
    });
}

// Exact windowed LD scores with covariates (winldcore.cpp:340-366 and
// :783-931): the genotypes of each partner range are projected,
// X <- (I - C R) X, and restandardized over the N rows (ddof 0), so r is no
// longer an integer Gram: dense FP64 panels and FP64 Gram products per chunk
// of rows, then the masked f(r) annotation sums.
static void window_ld_cov_impl(Context& c, const Prepared& P, int64_t row0, int64_t row1,
                               const int64_t* lo, const int64_t* hi, const double* annot,
                               int64_t K, double corr_dim, const DevCov& cv, double* out,
                               int64_t ld_row, int64_t ld_col) {
    const int64_t m = row1 - row0, N = P.g.N;
    if (K > window_cov_max_bins())
        fail(LDS_ERR_ARG, "at most %d annotation columns with covariates", window_cov_max_bins());
    DevBuf dann, dlo, dhi, dout, dX, dS, dtmp;
    double* an = dann.as<double>((size_t)(m * K));
    h2d(an, annot, (size_t)(m * K), c.st);
    int64_t* dl = dlo.as<int64_t>((size_t)m);
    int64_t* dh = dhi.as<int64_t>((size_t)m);
    h2d(dl, lo, (size_t)m, c.st);
    h2d(dh, hi, (size_t)m, c.st);
    double* o = dout.as<double>((size_t)(m * K));
    ck(cudaMemsetAsync(o, 0, sizeof(double) * (size_t)(m * K), c.st), "memset");
    const double corr_den = corr_dim > 0.0 ? 1.0 / (corr_dim - 1.0) : 0.0;
    constexpr int64_t T = 2048;
    for (int64_t j0 = row0; j0 < row1; j0 += T) {
        const int64_t j1 = std::min(row1, j0 + T);
        int64_t p0 = j0, p1 = j1;
        for (int64_t j = j0; j < j1; ++j) {
            if (hi[j - row0] <= lo[j - row0]) continue;
            p0 = std::min(p0, lo[j - row0]);
            p1 = std::max(p1, hi[j - row0]);
        }
        const int64_t Pn = p1 - p0, rows = j1 - j0;
        double* X = dX.as<double>((size_t)(N * Pn));
        launch_decode_standardized(P.g, p0, Pn, static_cast<const double*>(P.d_mean.p),
                                   static_cast<const double*>(P.d_sdinv.p), X, N, c.st);
        project_cols(c, X, N, Pn, cv, false, dtmp);
        launch_restandardize_cols(X, N, N, Pn, c.st);
        double* S = dS.as<double>((size_t)(rows * Pn));
        DGemmArgs a;
        a.M = rows;
        a.N = Pn;
        a.K = N;
        a.A = X + (j0 - p0) * N;  // X^T rows of the chunk
        a.a_ms = N;
        a.a_ks = 1;
        a.B = X;
        a.b_ks = 1;
        a.b_ns = N;
        a.C = S;
        a.c_ms = 1;
        a.c_ns = rows;
        launch_dgemm(a, c.st);
        launch_window_cov_epilogue(S, rows, p0, dl + (j0 - row0), dh + (j0 - row0), an, row0,
                                   (int)K, 1.0 / (double)N, corr_den, o + (j0 - row0) * K, c.st);
        ck(cudaGetLastError(), "windowed LD with covariates");
        ck(cudaStreamSynchronize(c.st), "windowed LD with covariates");  // X, S are reused
    }
    std::vector<double> h((size_t)(m * K));
    d2h(h.data(), o, h.size(), c.st);
    ck(cudaStreamSynchronize(c.st), "windowed LD with covariates");
    for (int64_t r = 0; r < m; ++r)
        for (int64_t b = 0; b < K; ++b) out[r * ld_row + b * ld_col] = h[(size_t)(r * K + b)];
}

LDS_API int lds_compute_windowed_ld_chr(const char* bed_prefix, const char* fam_path,
                                        int chr_start, int chr_end, const int64_t* bp,
                                        const double* annot_chr, int64_t K, double ld_wind_kb,
                                        int chunk_size, const int64_t* row_sel, int64_t n_row_sel,
                                        const double* C, const double* R, int64_t p,
                                        int impute_mode, int has_impute_seed,
                                        uint64_t impute_seed, int panel_cols, int cache_mb,
                                        double* out) {
    return guarded([&] {
        (void)panel_cols;  // CPU panel/cache tiling knobs: the result does not depend on them
        (void)cache_mb;
        if (chr_end < chr_start) fail(LDS_ERR_ARG, "chr_end must be >= chr_start");
        const int64_t m = (int64_t)chr_end - chr_start;
        if (m <= 0) fail(LDS_ERR_ARG, "Chromosome slice is empty");
        if (chunk_size <= 0) fail(LDS_ERR_ARG, "chunk_size must be > 0");
        const double window_bp = ld_wind_kb * 1000.0;
        if (!std::isfinite(window_bp) || window_bp <= 0.0)
            fail(LDS_ERR_ARG, "ld_wind_kb must define a finite positive BP window");
        if (!bp || !annot_chr || !out) fail(LDS_ERR_ARG, "null argument");
        for (int64_t i = 1; i < m; ++i)
            if (bp[i] < bp[i - 1])
                fail(LDS_ERR_ARG, "BP not sorted within chromosome block. Sort your .bim by CHR+BP.");
        if (K <= 0) fail(LDS_ERR_ARG, "annot_chr must have at least one column");
        if (impute_mode != LDS_IMPUTE_MEAN && impute_mode != LDS_IMPUTE_HWE)
            fail(LDS_ERR_ARG, "impute_mode must be 'mean' or 'hwe'");
        const bool cov = C && R && p > 0;
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        int64_t M_total = 0;
        Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel, impute_mode,
                                        has_impute_seed ? impute_seed : 0ULL, 0, &M_total);
        if (chr_start < 0 || chr_end > P.g.M)
            fail(LDS_ERR_IO, "BED file too small for requested block: %s.bed", bed_prefix);
        if (P.g.N <= 2) fail(LDS_ERR_ARG, "Too few rows for windowed LD score computation");
        const double corr_dim = (double)(P.g.N - (cov ? p : 1));
        if (corr_dim <= 1.0)
            fail(LDS_ERR_ARG, "Too few residual dimensions for unbiased windowed r^2 correction");
        // Partner interval of SNP j: |bp_i - bp_j| <= W (winldcore.cpp:434-442), a
        // contiguous run of the sorted positions.
        std::vector<int64_t> lo((size_t)m), hi((size_t)m);
        int64_t a = 0, b = 0;
        for (int64_t j = 0; j < m; ++j) {
            while (a < j && std::fabs((long double)bp[j] - (long double)bp[a]) > (long double)window_bp) ++a;
            if (b < j + 1) b = j + 1;
            while (b < m && std::fabs((long double)bp[b] - (long double)bp[j]) <= (long double)window_bp) ++b;
            lo[(size_t)j] = chr_start + a;
            hi[(size_t)j] = chr_start + b;
        }
        std::vector<double> ann((size_t)(m * K));
        for (int64_t j = 0; j < m; ++j)
            for (int64_t k = 0; k < K; ++k) ann[(size_t)(j * K + k)] = annot_chr[k * m + j];
        if (cov) {
            DevCov cv;
            upload_cov<double>(c, cv, C, R, P.g.N, p);
            window_ld_cov_impl(c, P, chr_start, chr_end, lo.data(), hi.data(), ann.data(), K,
                               corr_dim, cv, out, 1, m);
            return;
        }
        window_ld_impl(c, P, chr_start, chr_end, lo.data(), hi.data(), ann.data(), K, corr_dim, out,
                       1, m);
    });
}

// Minor allele frequency per SNP over the selected samples (compute_maf_block,
// genotype.cpp:1634-1730): p = sum / (2 nobs) clipped to [0, 1], maf = min(p, 1 - p).
LDS_API int lds_compute_maf_bed(const char* bed_prefix, const char* fam_path, int nsnps,
                                int step_size, const int64_t* row_sel, int64_t n_row_sel,
                                double* maf_out) {
    return guarded([&] {
        if (nsnps < 0) fail(LDS_ERR_ARG, "nsnps must be >= 0");
        if (step_size <= 0) fail(LDS_ERR_ARG, "step_size must be > 0");
        if (row_sel && n_row_sel <= 0) fail(LDS_ERR_ARG, "No rows selected in compute_maf_bed");
        if (nsnps == 0) return;
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        Prepared& P = prepared_for_file(c, bed_prefix, fam_path, row_sel, n_row_sel,
                                        LDS_IMPUTE_MEAN, 0ULL, 1, nullptr);
        if (nsnps > P.g.M)
            fail(LDS_ERR_IO, "BED file too small for requested block: %s.bed", bed_prefix);
        for (int64_t j = 0; j < nsnps; ++j) {
            const SnpCounts& k = P.counts[(size_t)j];
            const long long nobs = (long long)k.n[0] + k.n[1] + k.n[2];
            const long long sum = (long long)k.n[1] + 2LL * k.n[2];
            double pp = 0.0;
            if (nobs > 0) {
                pp = (double)sum / (2.0 * (double)nobs);
                if (pp < 0.0) pp = 0.0;
                if (pp > 1.0) pp = 1.0;
            }
            maf_out[j] = std::min(pp, 1.0 - pp);
        }
    });
}

LDS_API int lds_nn_band(int64_t geno, int D, double* xx_out, int32_t* counts_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        if (D < 0 || D > LDS_NN_BAND_MAX) fail(LDS_ERR_ARG, "band width D must be in [0, 15]");
        Prepared& P = *it->second;
        const int64_t M = P.g.M, n = M * (D + 1);
        DevBuf dc, dx;
        int32_t* cnt = dc.as<int32_t>((size_t)(n * 4));
        double* xx = dx.as<double>((size_t)n);
        launch_nn_band(P.g, D, cnt, c.st);
        launch_nn_band_finish(M, D, cnt, static_cast<double*>(P.d_mean.p),
                              static_cast<double*>(P.d_sdinv.p), xx, c.st);
        ck(cudaGetLastError(), "launch");
        if (xx_out) d2h(xx_out, xx, (size_t)n, c.st);
        if (counts_out) d2h(counts_out, cnt, (size_t)(n * 4), c.st);
        ck(cudaStreamSynchronize(c.st), "band sync");
    });
}

LDS_API int lds_gw_plan_create(int64_t geno, const double* annot, int64_t K, int nvecs,
                               int step_size, int vtile, uint64_t seed, int rand_dist,
                               double resvar_eps, int as_float, int with_mc, int64_t* plan_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        auto pl = plan_create(c, it->second, annot, K, nvecs, step_size, vtile, seed, rand_dist,
                              resvar_eps, as_float, with_mc);
        const int64_t h = next_handle();
        plan_table()[h] = std::move(pl);
        *plan_out = h;
    });
}

static GwPlan& plan_of(int64_t h) {
    auto it = plan_table().find(h);
    if (it == plan_table().end()) fail(LDS_ERR_ARG, "unknown plan handle");
    return *it->second;
}

LDS_API int lds_gw_plan_create_shard(int64_t geno, const double* annot, int64_t K, int nvecs,
                                     int step_size, int vtile, uint64_t seed, int rand_dist,
                                     double resvar_eps, int as_float, int with_mc,
                                     int64_t snp_offset, int64_t* plan_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        if (snp_offset != 0 && it->second->impute == LDS_IMPUTE_HWE)
            fail(LDS_ERR_ARG, "HWE imputation seeds by the SNP's index in the fileset; build SNP "
                              "shards with impute_mode 'mean'");
        auto pl = plan_create(c, it->second, annot, K, nvecs, step_size, vtile, seed, rand_dist,
                              resvar_eps, as_float, with_mc, snp_offset);
        const int64_t h = next_handle();
        plan_table()[h] = std::move(pl);
        *plan_out = h;
    });
}

LDS_API int lds_gw_plan_tiles(int64_t plan, int* n_tiles, int* tile_sizes, int64_t* sketch_rows) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        if (n_tiles) *n_tiles = (int)pl.tiles.size();
        if (tile_sizes)
            for (size_t t = 0; t < pl.tiles.size(); ++t) tile_sizes[t] = pl.tiles[t]->V;
        if (sketch_rows) *sketch_rows = pl.P->g.N_pad;
    });
}

LDS_API int lds_gw_plan_phase1(int64_t plan, int tile, double* d_sketch) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        if (tile < 0 || tile >= (int)pl.tiles.size()) fail(LDS_ERR_ARG, "V-tile index out of range");
        if (!d_sketch) fail(LDS_ERR_ARG, "sketch buffer is NULL");
        if (tile == 0) plan_zero(c, pl);
        int e = 0;
        plan_enqueue_phase1(c, pl, (size_t)tile, d_sketch, nullptr, e);
        ck(cudaGetLastError(), "launch");
    });
}

LDS_API int lds_gw_plan_phase2(int64_t plan, int tile, const double* d_sketch) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        if (tile < 0 || tile >= (int)pl.tiles.size()) fail(LDS_ERR_ARG, "V-tile index out of range");
        if (!d_sketch) fail(LDS_ERR_ARG, "sketch buffer is NULL");
        int e = 0;
        plan_enqueue_phase2(c, pl, (size_t)tile, d_sketch, nullptr, e);
        ck(cudaGetLastError(), "launch");
    });
}

LDS_API int lds_gw_plan_set_bin_totals(int64_t plan, const double* Mk) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        for (int64_t k = 0; k < pl.K; ++k) pl.Mk[(size_t)k] = Mk[k];
    });
}

LDS_API int lds_gw_plan_bin_totals(int64_t plan, double* Mk) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        for (int64_t k = 0; k < pl.K; ++k) Mk[k] = pl.Mk[(size_t)k];
    });
}

LDS_API int lds_gw_plan_execute(int64_t plan) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        plan_execute(c, plan_of(plan));
    });
}

LDS_API int lds_gw_plan_results(int64_t plan, double* ldscore, double* meansq_accum,
                                double* inv_out, double* mc_aggregate_sumsq,
                                double* mc_per_snp_sumsq) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        plan_results(c, plan_of(plan), ldscore, meansq_accum, inv_out, mc_aggregate_sumsq,
                     mc_per_snp_sumsq);
    });
}

LDS_API int lds_gw_plan_set_checks(int64_t plan, int on) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        if (pl.executed) fail(LDS_ERR_ARG, "set the product checks before the plan's first execute");
        if (on && !pl.umma) fail(LDS_ERR_ARG, "product checks need the tcgen05 phase-2 kernel");
        pl.check = on ? 1 : 0;
        if (!pl.check) return;
        const int64_t M = pl.P->g.M;
        pl.chk_lhs.as<unsigned long long>(2 * (size_t)M);
        pl.chk_rhs.as<unsigned long long>(2 * (size_t)M);
        pl.chk_u.as<unsigned long long>((size_t)pl.P->g.N_pad);
        std::vector<int4> tiles;
        for (int64_t j = 0; j < M; j += 128) tiles.push_back(make_int4((int)j, (int)M, 0, 0));
        pl.chk_ntiles = (int64_t)tiles.size();
        h2d(pl.chk_tiles.as<int4>(tiles.size()), tiles.data(), tiles.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "check tiles");
    });
}

LDS_API int lds_gw_plan_check(int64_t plan, unsigned long long* lhs, unsigned long long* rhs,
                              int64_t* mismatches, int64_t* first_snp, double* check_ms) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        if (!pl.check) fail(LDS_ERR_ARG, "product checks are off for this plan (lds_gw_plan_set_checks)");
        if (!pl.executed) fail(LDS_ERR_ARG, "no estimate of this plan has run");
        const size_t n = 2 * (size_t)pl.P->g.M;
        std::vector<unsigned long long> hl, hr;
        if (!lhs) { hl.resize(n); lhs = hl.data(); }
        if (!rhs) { hr.resize(n); rhs = hr.data(); }
        ck(cudaStreamSynchronize(c.st), "sync");
        plan_kernel_times(pl);
        d2h(lhs, static_cast<unsigned long long*>(pl.chk_lhs.p), n, c.st);
        d2h(rhs, static_cast<unsigned long long*>(pl.chk_rhs.p), n, c.st);
        ck(cudaStreamSynchronize(c.st), "checksums");
        const int64_t bad = count_check_mismatches(lhs, rhs, (int64_t)(n / 2), first_snp);
        if (mismatches) *mismatches = bad;
        if (check_ms) *check_ms = pl.check_ms;
    });
}

LDS_API int lds_gw_plan_kernel_ms(int64_t plan, double* ms4) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GwPlan& pl = plan_of(plan);
        ck(cudaStreamSynchronize(c.st), "sync");
        plan_kernel_times(pl);
        for (int i = 0; i < 4; ++i) ms4[i] = pl.kernel_ms[i];
    });
}

LDS_API int lds_gw_plan_destroy(int64_t plan) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.ready) ck(cudaStreamSynchronize(c.st), "sync");
        plan_table().erase(plan);
    });
}

LDS_API int lds_debug_xt_products_umma(const uint8_t* bed_rows, int64_t bed_row_bytes,
                                       int64_t n, int64_t L, const int8_t* y, int64_t V,
                                       int64_t* out_g, int64_t* out_o) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (L <= 0 || V <= 0 || n <= 0) fail(LDS_ERR_ARG, "invalid sizes");
        auto P = prepare(c, bed_rows, bed_row_bytes, n, L, nullptr, 0, LDS_IMPUTE_MEAN, 0, 1,
                         "debug");
        const int64_t Np = P->g.N_pad;
        const int nc = umma::ncolp_for((int)V);
        std::vector<int8_t> yq((size_t)(nc * Np), 0);
        for (int64_t q = 0; q < 4 * V; ++q)
            for (int64_t i = 0; i < n; ++i) yq[(size_t)umma::digit_offset(q, i, nc)] = y[q * n + i];
        DevBuf dyq, rg, ro, st;
        int8_t* d_yq = dyq.as<int8_t>(yq.size());
        h2d(d_yq, yq.data(), yq.size(), c.st);
        long long* dg = rg.as<long long>((size_t)(L * V));
        long long* dO = ro.as<long long>((size_t)(L * V));
        unsigned* dst = st.as<unsigned>(1);
        ck(cudaMemsetAsync(dst, 0, 4, c.st), "memset");
        const CUtensorMap tA = make_map_2d(P->g.codes, (uint64_t)P->g.nbp, (uint64_t)P->g.M_pad,
                                           (uint64_t)P->g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
        umma::P2UArgs u;
        u.yq = d_yq;
        u.yq_cols = nc;
        u.K = 1;
        u.V = (int)V;
        u.ncolp = nc;
        u.ngroups = (nc + 255) / 256;
        u.box_rows = std::min(256, nc);
        u.nkt = (int)(Np / 128);
        u.M = L;
        u.j0 = 0;
        u.j1 = L;
        u.out_row0 = 0;
        u.mean = static_cast<double*>(P->d_mean.p);
        u.sdinv = static_cast<double*>(P->d_sdinv.p);
        u.status = dst;
        u.raw_g = dg;
        u.raw_o = dO;
        umma::launch_p2_umma(tA, u, c.st);
        ck(cudaGetLastError(), "launch");
        unsigned stv = 0;
        d2h(&stv, dst, 1, c.st);
        d2h(reinterpret_cast<long long*>(out_g), dg, (size_t)(L * V), c.st);
        d2h(reinterpret_cast<long long*>(out_o), dO, (size_t)(L * V), c.st);
        ck(cudaStreamSynchronize(c.st), "debug umma products");
        if (stv) fail(LDS_ERR_CUDA, "phase-2 tensor-core pipeline wait timed out (code %u)", stv);
    });
}

LDS_API int lds_set_p2_kernel(int impl) {
    if (impl != 0 && impl != 1) {
        g_err = "p2 kernel must be 0 (mma.sync) or 1 (tcgen05)";
        return LDS_ERR_ARG;
    }
    p2_impl() = impl;
    return LDS_OK;
}

LDS_API int lds_win_plan_create(int64_t geno, const double* annot, int64_t K,
                                const int64_t* window_starts, int64_t n_windows, int nvecs,
                                int step_size, int vtile, uint64_t seed, int rand_dist,
                                double resvar_eps, int as_float, int with_mc, double batch_gb,
                                int64_t* plan_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
        auto pl = win_plan_create(c, it->second, annot, K, window_starts, n_windows, nvecs,
                                  step_size, vtile, seed, rand_dist, resvar_eps, as_float, with_mc,
                                  batch_gb > 0 ? batch_gb : 8.0);
        const int64_t h = next_handle();
        win_table()[h] = std::move(pl);
        *plan_out = h;
    });
}

LDS_API int lds_win_ldscore(const uint8_t* bed_rows, int64_t bed_row_bytes, int64_t n_total,
                            int64_t M, const int64_t* row_sel, int64_t n_row_sel,
                            const double* annot, int64_t K, const int64_t* window_starts,
                            int64_t n_windows, int nvecs, int step_size, int vtile, uint64_t seed,
                            int rand_dist, int ddof, int impute_mode, uint64_t impute_seed,
                            double resvar_eps, int as_float, int n_chunks, int p1_sb_per_cta,
                            double* ldscore, double* meansq_accum, double* inv_out) {
    return guarded([&] {
        win_ldscore_impl(bed_rows, bed_row_bytes, n_total, M, row_sel, n_row_sel, annot, K,
                         window_starts, n_windows, nvecs, step_size, vtile, seed, rand_dist, ddof,
                         impute_mode, impute_seed, resvar_eps, as_float, n_chunks, p1_sb_per_cta,
                         ldscore, meansq_accum, inv_out);
    });
}

static WinPlan& win_of_handle(int64_t h) {
    auto it = win_table().find(h);
    if (it == win_table().end()) fail(LDS_ERR_ARG, "unknown windowed plan handle");
    return *it->second;
}

LDS_API int lds_win_plan_execute(int64_t plan) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        win_execute(c, win_of_handle(plan));
    });
}

LDS_API int lds_win_plan_results(int64_t plan, double* ldscore, double* meansq_accum,
                                 double* inv_out, double* mc_per_snp_sumsq) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        win_results(c, win_of_handle(plan), ldscore, meansq_accum, inv_out, mc_per_snp_sumsq);
    });
}

LDS_API int lds_win_plan_kernel_ms(int64_t plan, double* ms4) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        ck(cudaStreamSynchronize(c.st), "sync");
        win_times(pl);
        for (int i = 0; i < 4; ++i) ms4[i] = pl.kernel_ms[i];
    });
}

LDS_API int lds_win_plan_set_tiling(int64_t plan, int p1_sb_per_cta) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        if (pl.graph) fail(LDS_ERR_ARG, "set the tiling before the plan's first execute");
        if (p1_sb_per_cta < 0 || p1_sb_per_cta > 4096)
            fail(LDS_ERR_ARG, "p1_sb_per_cta must be in [0, 4096]");
        pl.p1_spc = p1_sb_per_cta;
    });
}

LDS_API int lds_win_plan_set_p2_order(int64_t plan, int bin_chunk) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        if (pl.graph) fail(LDS_ERR_ARG, "set the phase-2 order before the plan's first execute");
        if (bin_chunk < 0 || bin_chunk > 4096) fail(LDS_ERR_ARG, "bin_chunk must be in [0, 4096]");
        pl.p2_chunk = bin_chunk;
        for (auto& b : pl.batches) build_win_work(c, pl, b);
        ck(cudaStreamSynchronize(c.st), "phase-2 order");
    });
}

LDS_API int lds_win_plan_set_p2_bins(int64_t plan, int bins_per_cta) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        if (pl.graph) fail(LDS_ERR_ARG, "set the phase-2 bins per CTA before the plan's first execute");
        if (bins_per_cta < 0 || bins_per_cta > 4096)
            fail(LDS_ERR_ARG, "bins_per_cta must be in [0, 4096]");
        pl.p2_nb = bins_per_cta;
        for (auto& b : pl.batches) build_win_work(c, pl, b);
        ck(cudaStreamSynchronize(c.st), "phase-2 bins per CTA");
    });
}

LDS_API int lds_win_plan_set_checks(int64_t plan, int on) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        if (pl.graph) fail(LDS_ERR_ARG, "set the product checks before the plan's first execute");
        pl.check = on ? 1 : 0;
        if (pl.check) {
            const size_t M = (size_t)pl.P->g.M;
            int64_t maxw = 1;
            for (const auto& b : pl.batches) maxw = std::max(maxw, b.w1 - b.w0);
            pl.chk_lhs.as<unsigned long long>(2 * M);
            pl.chk_rhs.as<unsigned long long>(2 * M);
            pl.chk_u.as<unsigned long long>((size_t)maxw * (size_t)pl.P->g.N_pad);
        }
        // one more event per (V-tile, batch) closes the check interval
        const size_t need = 1 + (size_t)pl.ev_per() * pl.vt.size() * pl.batches.size();
        while (pl.ev.size() < need) {
            cudaEvent_t e = nullptr;
            ck(cudaEventCreate(&e), "event");
            pl.ev.push_back(e);
        }
        while (pl.ev.size() > need) {
            cudaEventDestroy(pl.ev.back());
            pl.ev.pop_back();
        }
    });
}

LDS_API int lds_win_plan_check(int64_t plan, unsigned long long* lhs, unsigned long long* rhs,
                               int64_t* mismatches, int64_t* first_snp, double* check_ms) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        if (!pl.check) fail(LDS_ERR_ARG, "product checks are off for this plan (lds_win_plan_set_checks)");
        if (!pl.graph) fail(LDS_ERR_ARG, "no estimate of this plan has run");
        const size_t n = 2 * (size_t)pl.P->g.M;
        std::vector<unsigned long long> hl, hr;
        if (!lhs) { hl.resize(n); lhs = hl.data(); }
        if (!rhs) { hr.resize(n); rhs = hr.data(); }
        ck(cudaStreamSynchronize(c.st), "sync");
        win_times(pl);
        d2h(lhs, static_cast<unsigned long long*>(pl.chk_lhs.p), n, c.st);
        d2h(rhs, static_cast<unsigned long long*>(pl.chk_rhs.p), n, c.st);
        ck(cudaStreamSynchronize(c.st), "checksums");
        const int64_t bad = count_check_mismatches(lhs, rhs, (int64_t)(n / 2), first_snp);
        if (mismatches) *mismatches = bad;
        if (check_ms) *check_ms = pl.kernel_ms[4];
    });
}

LDS_API int lds_check_vectors(const unsigned long long* lhs, const unsigned long long* rhs,
                              int64_t n_snps, int64_t* mismatches, int64_t* first_snp) {
    return guarded([&] {
        if (n_snps < 0 || (n_snps > 0 && (!lhs || !rhs))) fail(LDS_ERR_ARG, "invalid checksum vectors");
        const int64_t bad = count_check_mismatches(lhs, rhs, n_snps, first_snp);
        if (mismatches) *mismatches = bad;
    });
}

LDS_API int lds_win_plan_cv_annot(int64_t plan, const double** d_annot) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        const WinPlan& pl = win_of_handle(plan);
        if (!d_annot) fail(LDS_ERR_ARG, "null output");
        if (!pl.annot_d.p) fail(LDS_ERR_ARG, "plan has no control-variate inputs (lds_win_plan_set_cv)");
        ck(cudaStreamSynchronize(c.st), "sync");  // the upload is complete for other streams
        *d_annot = static_cast<const double*>(pl.annot_d.p);
    });
}

LDS_API int lds_win_plan_bin_totals(int64_t plan, double* mkw_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        const WinPlan& pl = win_of_handle(plan);
        if (!mkw_out) fail(LDS_ERR_ARG, "null output");
        std::memcpy(mkw_out, pl.Mkw.data(), sizeof(double) * pl.Mkw.size());
    });
}

LDS_API int lds_win_plan_set_cv(int64_t plan, const double* annot, int split_tiles, int band_D) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        win_set_cv(c, win_of_handle(plan), annot, split_tiles, band_D);
    });
}

LDS_API int lds_win_plan_tiles(int64_t plan, int* n_tiles, int* tile_sizes) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        *n_tiles = (int)pl.vt.size();
        if (tile_sizes)
            for (size_t t = 0; t < pl.vt.size(); ++t) tile_sizes[t] = pl.vt[t];
    });
}

LDS_API int lds_win_plan_cv_outputs(int64_t plan, int device_ptrs, double* meansq_tiles,
                                    double* C_tiles, double* mu, double* xx) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        const int64_t M = pl.P->g.M, K = pl.K;
        const size_t nout = (size_t)(M * K) * (size_t)pl.ntiles_out();
        const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        auto cp = [&](double* dst, const DevBuf& src, size_t n) {
            if (dst && n) ck(cudaMemcpyAsync(dst, src.p, n * sizeof(double), kind, c.st), "copy");
        };
        unsigned st = 0;
        d2h(&st, static_cast<unsigned*>(pl.status.p), 1, c.st);
        cp(meansq_tiles, pl.accum, nout);
        if (pl.cv_D > 0) {
            cp(C_tiles, pl.cvC, nout);
            cp(mu, pl.cvMu, (size_t)(M * K));
            cp(xx, pl.xx, (size_t)(M * (pl.cv_D + 1)));
        } else if (C_tiles || mu || xx) {
            fail(LDS_ERR_ARG, "plan has no control-variate outputs (lds_win_plan_set_cv)");
        }
        ck(cudaStreamSynchronize(c.st), "cv outputs");
        if (st) fail(LDS_ERR_CUDA, "tensor-core pipeline wait timed out (code %u)", st);
        win_times(pl);
    });
}

LDS_API int lds_win_plan_cv_ms(int64_t plan, double* ms) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        WinPlan& pl = win_of_handle(plan);
        ck(cudaStreamSynchronize(c.st), "sync");
        win_times(pl);
        *ms = pl.cv_ms;
    });
}

// ---------------------------------------------------------------------------
// Surrogate network (learned control variate); device pointers owned by the caller.
// ---------------------------------------------------------------------------
static void check_mlp_dims(int in_dim, int out_dim) {
    if (in_dim < 1 || in_dim > LDS_MLP_MAX_IN || out_dim < 1 || out_dim > LDS_MLP_MAX_OUT)
        fail(LDS_ERR_ARG, "network input width must be in [1, 128] and output width in [1, 64]");
}

LDS_API int64_t lds_mlp_param_count(int in_dim, int out_dim) {
    return mlp_layout(in_dim, out_dim).total;
}

LDS_API int lds_mlp_forward(const float* d_params, int in_dim, int out_dim, const float* d_x,
                            int64_t n, float* d_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        check_mlp_dims(in_dim, out_dim);
        MlpArgs a;
        a.params = d_params;
        a.in = in_dim;
        a.out = out_dim;
        void* pack = c.mlp_pack.as<uint16_t>(mlp_pack_elems(in_dim, out_dim));
        launch_mlp_pack(a, pack, c.st);
        launch_mlp_forward(a, pack, d_x, nullptr, n, nullptr, d_out, nullptr, nullptr, nullptr, 0.f,
                           c.st);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(c.st), "mlp forward");
    });
}

LDS_API int lds_mlp_loss_grad(const float* d_params, int in_dim, int out_dim, const float* d_x,
                              const float* d_t, int64_t n, float* d_grad, double* loss_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        check_mlp_dims(in_dim, out_dim);
        if (n <= 0) fail(LDS_ERR_ARG, "n must be positive");
        MlpArgs a;
        a.params = d_params;
        a.in = in_dim;
        a.out = out_dim;
        const int op = mlp_out_pad(out_dim);
        const int64_t P = mlp_layout(in_dim, out_dim).total;
        float* z = c.mlp_zs.as<float>((size_t)(n * 3 * kMlpHidden));
        float* dz = c.mlp_dzs.as<float>((size_t)(n * 3 * kMlpHidden));
        float* d = c.mlp_dout.as<float>((size_t)(n * op));
        double* l = c.mlp_loss.as<double>(1);
        ck(cudaMemsetAsync(l, 0, sizeof(double), c.st), "memset");
        ck(cudaMemsetAsync(d_grad, 0, sizeof(float) * (size_t)P, c.st), "memset");
        void* pack = c.mlp_pack.as<uint16_t>(mlp_pack_elems(in_dim, out_dim));
        launch_mlp_pack(a, pack, c.st);
        launch_mlp_forward(a, pack, d_x, nullptr, n, d_t, nullptr, z, d, l,
                           1.0f / (float)(n * out_dim), c.st);
        launch_mlp_backward(a, pack, d_x, nullptr, n, z, d, dz, d_grad, c.st);
        ck(cudaGetLastError(), "launch");
        if (loss_out) d2h(loss_out, l, 1, c.st);
        ck(cudaStreamSynchronize(c.st), "mlp grad");
    });
}

LDS_API int lds_mlp_train(float* d_params, int in_dim, int out_dim, const float* d_x,
                          const float* d_t, int64_t n, int epochs, int batch, float lr,
                          uint64_t seed, double* loss_per_epoch) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        check_mlp_dims(in_dim, out_dim);
        if (n <= 0 || epochs < 0 || batch <= 0) fail(LDS_ERR_ARG, "invalid training sizes");
        MlpArgs a;
        a.params = d_params;
        a.in = in_dim;
        a.out = out_dim;
        const int op = mlp_out_pad(out_dim);
        const int64_t P = mlp_layout(in_dim, out_dim).total;
        const int64_t B = std::min<int64_t>(batch, n);
        float* dm = c.mlp_m.as<float>((size_t)P);
        float* dv = c.mlp_v.as<float>((size_t)P);
        float* dg = c.mlp_g.as<float>((size_t)P);
        float* z = c.mlp_zs.as<float>((size_t)(B * 3 * kMlpHidden));
        float* dz = c.mlp_dzs.as<float>((size_t)(B * 3 * kMlpHidden));
        float* d = c.mlp_dout.as<float>((size_t)(B * op));
        double* l = c.mlp_loss.as<double>((size_t)std::max(epochs, 1));
        ck(cudaMemsetAsync(dm, 0, sizeof(float) * (size_t)P, c.st), "memset");
        ck(cudaMemsetAsync(dv, 0, sizeof(float) * (size_t)P, c.st), "memset");
        ck(cudaMemsetAsync(l, 0, sizeof(double) * (size_t)std::max(epochs, 1), c.st), "memset");
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        // All epochs' shuffles up front: one upload, no host round trip per epoch.
        std::vector<int32_t> perm((size_t)(n * std::max(epochs, 1)));
        std::mt19937_64 rng(seed);
        for (int e = 0; e < epochs; ++e) {
            int32_t* pe = perm.data() + (size_t)e * (size_t)n;
            for (int64_t i = 0; i < n; ++i) pe[i] = (int32_t)i;
            std::shuffle(pe, pe + n, rng);
        }
        int32_t* r = c.mlp_rows.as<int32_t>(perm.size());
        h2d(r, perm.data(), perm.size(), c.st);
        void* pack = c.mlp_pack.as<uint16_t>(mlp_pack_elems(in_dim, out_dim));
        int64_t step = 0;
        const int64_t nsteps = (n + B - 1) / B;
        for (int e = 0; e < epochs; ++e) {
            const int32_t* re = r + (size_t)e * (size_t)n;
            for (int64_t s = 0; s < nsteps; ++s) {
                const int64_t nb = std::min<int64_t>(B, n - s * B);
                ck(cudaMemsetAsync(dg, 0, sizeof(float) * (size_t)P, c.st), "memset");
                launch_mlp_pack(a, pack, c.st);
                launch_mlp_forward(a, pack, d_x, re + s * B, nb, d_t, nullptr, z, d, l + e,
                                   1.0f / (float)(nb * out_dim * nsteps), c.st);
                launch_mlp_backward(a, pack, d_x, re + s * B, nb, z, d, dz, dg, c.st);
                ++step;
                // The loss scale folds 1/nsteps into the gradient (so the epoch's
                // loss sums to its mean); Adam is invariant to that scale except
                // through eps, which is scaled alike.
                launch_mlp_adam(d_params, dm, dv, dg, P, lr, b1, b2, eps * (float)(1.0 / nsteps),
                                1.0f - std::pow(b1, (float)step), 1.0f - std::pow(b2, (float)step),
                                c.st);
            }
        }
        ck(cudaGetLastError(), "launch");
        if (loss_per_epoch && epochs > 0) d2h(loss_per_epoch, l, (size_t)epochs, c.st);
        ck(cudaStreamSynchronize(c.st), "mlp train");
    });
}

LDS_API int lds_win_plan_destroy(int64_t plan) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.ready) ck(cudaStreamSynchronize(c.st), "sync");
        win_table().erase(plan);
    });
}

LDS_API uint64_t lds_window_seed(uint64_t root, int64_t w) { return window_seed(root, w); }

LDS_API int lds_debug_rademacher_block(uint64_t root, int blk_start, int v_start, int L, int V,
                                       double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (L <= 0 || V <= 0) fail(LDS_ERR_ARG, "invalid sizes");
        DevBuf dz;
        double* z = dz.as<double>((size_t)L * (size_t)V);
        device_rademacher(c, {ProbeUnit{0, L, 0, probe_seed(root, blk_start, v_start)}}, V, z, L);
        d2h(out, z, (size_t)L * (size_t)V, c.st);
        ck(cudaStreamSynchronize(c.st), "probe block");
    });
}

LDS_API int lds_last_timings(double* ms_out, int n) {
    Context& c = ctx();
    for (int i = 0; i < n && i < 4; ++i) ms_out[i] = c.timings[i];
    return LDS_OK;
}

LDS_API int lds_synth_bed(int64_t n, int64_t M, uint64_t seed, const int64_t* t0,
                          const int64_t* t1, int missing, uint8_t* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        const int64_t nb = (n + 3) / 4;
        DevBuf dt0, dt1, dout;
        int64_t* a = dt0.as<int64_t>((size_t)M);
        int64_t* b = dt1.as<int64_t>((size_t)M);
        h2d(a, t0, (size_t)M, c.st);
        h2d(b, t1, (size_t)M, c.st);
        uint8_t* o = dout.as<uint8_t>((size_t)(nb * M));
        launch_synth(n, M, seed, a, b, missing, o, c.st);
        d2h(out, o, (size_t)(nb * M), c.st);
        ck(cudaStreamSynchronize(c.st), "synth");
    });
}


// ---------------------------------------------------------------------------
// SUMMIT-GxE C ABI (include/lds.h)
// ---------------------------------------------------------------------------
static GxeCtx& gxe_of(int64_t h) {
    auto it = gxe_table().find(h);
    if (it == gxe_table().end()) fail(LDS_ERR_ARG, "unknown GxE kernel handle");
    return *it->second;
}
static GxePair& gxe_pair_of(int64_t h) {
    auto it = gxe_pair_table().find(h);
    if (it == gxe_pair_table().end()) fail(LDS_ERR_ARG, "unknown GxE right-pair handle");
    return *it->second;
}

// The kernel's constructor state (MultiEnvironmentKernel, gxeldcore.cpp:
// 10281-10297) for N samples; P is the resident image its blocks come from,
// or null when the caller passes dense standardized genotype blocks.
static int gxe_create_impl(std::shared_ptr<Prepared> P, int64_t N, int64_t E,
                           const double* environments, int64_t r, const double* common_basis,
                           const double* directions, int64_t F, const double* feature_basis,
                           const int64_t* power_indices, const int64_t* power_offsets,
                           const int32_t* ranks, int annotation_bins, int64_t* handle_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!handle_out) fail(LDS_ERR_ARG, "null argument");
        if (N <= 2 || E <= 0 || F <= 0 || r < 0 || annotation_bins <= 0 || !environments ||
            !directions || !feature_basis || !power_indices || !power_offsets || !ranks ||
            (r > 0 && !common_basis))
            fail(LDS_ERR_ARG, "Multi-environment native kernel inputs have incompatible dimensions");
        if (power_offsets[0] != 0)
            fail(LDS_ERR_ARG, "Multi-environment native feature offsets do not span their buffers");
        auto g = std::make_unique<GxeCtx>();
        g->P = P;
        g->N = N;
        g->N_pad = P ? P->g.N_pad : round_up(N, kSamplePad);
        g->E = E;
        g->r = r;
        g->K = annotation_bins;
        g->ranks.assign(ranks, ranks + E);
        for (int64_t e = 0; e < E; ++e) {
            const int rk = ranks[e];
            if (rk <= 0 || rk >= N) fail(LDS_ERR_ARG, "Multi-environment native feature rank is invalid");
            for (int pw = 0; pw < 4; ++pw)
                if (power_offsets[4 * e + pw + 1] - power_offsets[4 * e + pw] != rk)
                    fail(LDS_ERR_ARG, "Multi-environment native power-index ranges are malformed");
        }
        h2d(g->env.as<double>((size_t)(N * E)), environments, (size_t)(N * E), c.st);
        if (r > 0) h2d(g->common.as<double>((size_t)(N * r)), common_basis, (size_t)(N * r), c.st);
        // [d_e, 1] per environment for the direction and mean projection
        std::vector<double> dones((size_t)(2 * N * E), 1.0);
        for (int64_t e = 0; e < E; ++e)
            std::memcpy(&dones[(size_t)(2 * e * N)], directions + e * N, sizeof(double) * (size_t)N);
        h2d(g->dirs_ones.as<double>(dones.size()), dones.data(), dones.size(), c.st);
        h2d(g->ranks_d.as<int32_t>((size_t)E), ranks, (size_t)E, c.st);
        std::vector<double> ones((size_t)std::max<int64_t>(P ? P->g.M : 1, 1), 1.0);
        h2d(g->ones_M.as<double>(ones.size()), ones.data(), ones.size(), c.st);
        g->basis0.resize((size_t)E);
        for (int64_t e = 0; e < E; ++e) {
            const int rk = ranks[e];
            std::vector<double> b((size_t)(N * rk));
            for (int a = 0; a < rk; ++a) {
                const int64_t col = power_indices[power_offsets[4 * e] + a];
                if (col < 0 || col >= F) fail(LDS_ERR_ARG, "Multi-environment native power index is out of range");
                std::memcpy(&b[(size_t)(a * N)], feature_basis + col * N, sizeof(double) * (size_t)N);
            }
            h2d(g->basis0[(size_t)e].as<double>(b.size()), b.data(), b.size(), c.st);
            ck(cudaStreamSynchronize(c.st), "gxe create");
        }
        ck(cudaStreamSynchronize(c.st), "gxe create");
        const int64_t h = next_handle();
        gxe_table()[h] = std::move(g);
        *handle_out = h;
    });
}

LDS_API int lds_gxe_create(int64_t geno, int64_t E, const double* environments, int64_t r,
                           const double* common_basis, const double* directions, int64_t F,
                           const double* feature_basis, const int64_t* power_indices,
                           const int64_t* power_offsets, const int32_t* ranks, int annotation_bins,
                           int64_t* handle_out) {
    std::shared_ptr<Prepared> P;
    {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = geno_table().find(geno);
        if (it == geno_table().end()) {
            set_last_error("unknown genotype handle");
            return LDS_ERR_ARG;
        }
        P = it->second;
    }
    return gxe_create_impl(P, P->g.N, E, environments, r, common_basis, directions, F,
                           feature_basis, power_indices, power_offsets, ranks, annotation_bins,
                           handle_out);
}

LDS_API int lds_gxe_create_dense(int64_t N, int64_t E, const double* environments, int64_t r,
                                 const double* common_basis, const double* directions, int64_t F,
                                 const double* feature_basis, const int64_t* power_indices,
                                 const int64_t* power_offsets, const int32_t* ranks,
                                 int annotation_bins, int64_t* handle_out) {
    return gxe_create_impl(nullptr, N, E, environments, r, common_basis, directions, F,
                           feature_basis, power_indices, power_offsets, ranks, annotation_bins,
                           handle_out);
}

// Generalized GxE packed products (generalized_gxe_variant.inc:1749-1988) on
// a resident mean-imputed image.  The reference's Mailman mean pack scales
// SNP j by inv_j = sqrt((N - ddof) / M2_j) (genotype.cpp:1115-1131) and its
// products use out = mu sum - raw over the packed allele counts, i.e. the
// negated standardized genotypes: source = -X' rhs (N x cols), target =
// -X'^T rhs (L x cols), X' = inv (g - mu) on observed calls, 0 on missing.
// The products run on the phase-1 and phase-2 tensor-core kernels with the
// image's scale s_j, rescaled per SNP by inv_j / s_j.
static std::vector<double> pack_scale_ratio(const Prepared& P, int64_t j0, int64_t j1) {
    std::vector<double> r((size_t)(j1 - j0));
    const long long denominator = P.g.N - (long long)P.ddof;
    for (int64_t j = j0; j < j1; ++j) {
        const SnpCounts& k = P.counts[(size_t)j];
        const long long nobs = (long long)k.n[0] + k.n[1] + k.n[2];
        const long long sum = (long long)k.n[1] + 2LL * k.n[2];
        const long long sumsq = (long long)k.n[1] + 4LL * k.n[2];
        double inv = 1.0;
        if (nobs > 0) {
            double m2 = (double)sumsq - (double)sum * (double)sum / (double)nobs;
            if (m2 < 0.0 && m2 > -1.0e-12) m2 = 0.0;
            if (denominator > 0 && m2 > 0.0) inv = std::sqrt((double)denominator / m2);
        }
        r[(size_t)(j - j0)] = inv / P.sdinv[(size_t)j];
    }
    return r;
}

static Prepared& generalized_image(int64_t geno, int64_t j0, int64_t j1, int64_t cols) {
    auto it = geno_table().find(geno);
    if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
    Prepared& P = *it->second;
    if (P.impute != LDS_IMPUTE_MEAN)
        fail(LDS_ERR_ARG, "generalized packed products need a mean-imputed genotype image");
    if (j0 < 0 || j1 > P.g.M || j1 <= j0 || cols <= 0)
        fail(LDS_ERR_ARG, "Generalized packed product is mis-sized");
    return P;
}

LDS_API int lds_generalized_source_product(int64_t geno, int64_t j0, int64_t j1,
                                           const double* rhs, int64_t cols, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        Prepared& P = generalized_image(geno, j0, j1, cols);
        const int64_t L = j1 - j0, N = P.g.N, Np = P.g.N_pad;
        const std::vector<double> ratio = pack_scale_ratio(P, j0, j1);
        std::vector<double> Z((size_t)(L * cols)), ones((size_t)L, 1.0);
        for (size_t i = 0; i < Z.size(); ++i) Z[i] = -rhs[i];
        const int Vp = (int)round_up(cols, kColTile);
        const Csr cs = build_csr<double>(ones.data(), ratio.data(), L, 1, j0, Vp, c.slices,
                                         kSnpStep, P.constant.data());
        run_phase1(c, P, cs, 1, (int)cols, Z.data(), L, L, j0);
        std::vector<double> y((size_t)(Np * cols));
        d2h(y.data(), static_cast<double*>(c.y.p), y.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "generalized source product");
        for (int64_t q = 0; q < cols; ++q)
            std::memcpy(out + q * N, &y[(size_t)(q * Np)], sizeof(double) * (size_t)N);
    });
}

LDS_API int lds_generalized_target_product(int64_t geno, int64_t j0, int64_t j1,
                                           const double* rhs, int64_t cols, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        Prepared& P = generalized_image(geno, j0, j1, cols);
        const int64_t L = j1 - j0, N = P.g.N;
        const std::vector<double> ratio = pack_scale_ratio(P, j0, j1);
        const std::vector<double> Y(rhs, rhs + N * cols);
        const std::vector<double> pr = snp_products(c, P, j0, j1, Y, cols);
        for (int64_t j = 0; j < L; ++j)
            for (int64_t q = 0; q < cols; ++q)
                out[q * L + j] = -ratio[(size_t)j] * pr[(size_t)(j * cols + q)];
    });
}

// ---------------------------------------------------------------------------
// Products of the generalized per-variant GxE two-pass estimator
// (generalized_gxe_pass1.py / _pass2.py) on the image's own standardized
// genotypes x_ij = s_j (g_ij - mu_j), 0 on a missing call (the decoded blocks
// its genotype operator returns).
// ---------------------------------------------------------------------------
static Prepared& product_image(int64_t geno, int64_t j0, int64_t j1, int64_t cols) {
    auto it = geno_table().find(geno);
    if (it == geno_table().end()) fail(LDS_ERR_ARG, "unknown genotype handle");
    Prepared& P = *it->second;
    if (j0 < 0 || j1 > P.g.M || j1 <= j0 || cols <= 0) fail(LDS_ERR_ARG, "genotype product is mis-sized");
    return P;
}

LDS_API int lds_geno_source_product(int64_t geno, int64_t j0, int64_t j1, const double* annot,
                                    int64_t K, const double* Z, int64_t B, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!Z || !out || (annot && K <= 0)) fail(LDS_ERR_ARG, "null or mis-sized product argument");
        const int64_t nb = annot ? K : 1;
        Prepared& P = product_image(geno, j0, j1, B * nb);
        const int64_t L = j1 - j0, N = P.g.N, Np = P.g.N_pad;
        if (annot)
            for (int64_t q = 0; q < L * K; ++q)
                if (!std::isfinite(annot[q]) || annot[q] < 0.0)
                    fail(LDS_ERR_ARG, "annotations must be finite and nonnegative");
        std::vector<double> ones((size_t)(L * nb), 1.0), unit((size_t)L, 1.0);
        const int Vp = (int)round_up(B, kColTile);
        const Csr cs = build_csr<double>(annot ? annot : ones.data(), unit.data(), L, nb, j0, Vp,
                                         c.slices, kSnpStep, P.constant.data());
        run_phase1(c, P, cs, nb, (int)B, Z, L, L, j0);
        std::vector<double> y((size_t)(Np * nb * B));
        d2h(y.data(), static_cast<double*>(c.y.p), y.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "genotype source product");
        for (int64_t q = 0; q < nb * B; ++q)
            std::memcpy(out + q * N, &y[(size_t)(q * Np)], sizeof(double) * (size_t)N);
    });
}

LDS_API int lds_geno_target_product(int64_t geno, int64_t j0, int64_t j1, const double* Y,
                                    int64_t cols, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!Y || !out) fail(LDS_ERR_ARG, "null product argument");
        Prepared& P = product_image(geno, j0, j1, cols);
        const int64_t L = j1 - j0, N = P.g.N;
        const std::vector<double> Yv(Y, Y + N * cols);
        const std::vector<double> pr = snp_products(c, P, j0, j1, Yv, cols);
        for (int64_t j = 0; j < L; ++j)
            for (int64_t q = 0; q < cols; ++q) out[q * L + j] = pr[(size_t)(j * cols + q)];
    });
}

LDS_API int lds_global_variant_probes(uint64_t root_seed, uint64_t namespace_key, int64_t v0,
                                      int64_t L, int64_t p0, int64_t B, double* out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!out || L <= 0 || B <= 0 || v0 < 0 || p0 < 0) fail(LDS_ERR_ARG, "invalid probe block");
        auto mix = [](uint64_t v) {
            v += 0x9E3779B97F4A7C15ULL;
            v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
            v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
            return v ^ (v >> 31);
        };
        const uint64_t root_state = mix(root_seed ^ namespace_key ^ 0x9E3779B97F4A7C15ULL);
        DevBuf d;
        double* dp = d.as<double>((size_t)(L * B));
        launch_global_probes(root_state, v0, L, p0, B, dp, c.st);
        ck(cudaGetLastError(), "launch");
        d2h(out, dp, (size_t)(L * B), c.st);
        ck(cudaStreamSynchronize(c.st), "probes");
    });
}

LDS_API int lds_generalized_component_diagonal(int64_t geno, int64_t j0, int64_t j1,
                                               const double* annot, int K, const double* basis,
                                               int Q, const double* fixed, int R,
                                               const double* coef, double* numerator) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!annot || !basis || !numerator || K <= 0 || Q <= 0 || R < 0 || (R > 0 && (!fixed || !coef)))
            fail(LDS_ERR_ARG, "invalid component-diagonal arguments");
        if (Q > kGenMaxQ || R > kGenMaxR)
            fail(LDS_ERR_ARG, "component diagonals support at most %d bases and %d fixed effects",
                 kGenMaxQ, kGenMaxR);
        Prepared& P = product_image(geno, j0, j1, 1);
        const int64_t L = j1 - j0, N = P.g.N;
        // pairs: diagonals first, then lexicographic off-diagonals; kernel
        // factor 1 on the diagonal, 2 off it (context/spec.py ContextPairIndex)
        std::vector<int> pq, pr;
        std::vector<double> kf;
        for (int q = 0; q < Q; ++q) { pq.push_back(q); pr.push_back(q); kf.push_back(1.0); }
        for (int q = 0; q < Q - 1; ++q)
            for (int r = q + 1; r < Q; ++r) { pq.push_back(q); pr.push_back(r); kf.push_back(2.0); }
        const int Pn = (int)pq.size(), C = K * Pn;
        DevBuf da, db, df, dc, dq, dr, dk, dn;
        double* a = da.as<double>((size_t)(L * K));
        double* b = db.as<double>((size_t)(N * Q));
        double* f = df.as<double>((size_t)std::max<int64_t>(N * R, 1));
        double* cf = dc.as<double>((size_t)std::max<int64_t>(L * Q * R, 1));
        int* qd = dq.as<int>((size_t)Pn);
        int* rd = dr.as<int>((size_t)Pn);
        double* kd = dk.as<double>((size_t)Pn);
        double* nm = dn.as<double>((size_t)(C * N));
        h2d(a, annot, (size_t)(L * K), c.st);
        h2d(b, basis, (size_t)(N * Q), c.st);
        if (R > 0) {
            h2d(f, fixed, (size_t)(N * R), c.st);
            h2d(cf, coef, (size_t)(L * Q * R), c.st);
        }
        h2d(qd, pq.data(), pq.size(), c.st);
        h2d(rd, pr.data(), pr.size(), c.st);
        h2d(kd, kf.data(), kf.size(), c.st);
        h2d(nm, numerator, (size_t)(C * N), c.st);
        launch_component_diag(P.g.codes, P.g.nbp, static_cast<double*>(P.d_mean.p),
                              static_cast<double*>(P.d_sdinv.p), j0, L, N, a, K, b, Q, f, R, cf,
                              qd, rd, kd, Pn, nm, c.st);
        ck(cudaGetLastError(), "launch");
        d2h(numerator, nm, (size_t)(C * N), c.st);
        ck(cudaStreamSynchronize(c.st), "component diagonal");
    });
}

// Pass 2 of the generalized estimator on the device; `fill` writes the
// right-hand side's K B F columns (N_pad samples each, rows past N zero) into
// the zeroed FP64 workspace Y.
static void gen_pass2_run(Context& c, int64_t geno,
                          const std::function<void(double* Y, int64_t N, int64_t Np)>& fill,
                          int K, int B, int F, int P, const int* term_off, const int* term_f1,
                          const int* term_f2, double residual_rank, const double* annot,
                          int64_t variant_block, double* directional, double* directed) {
    {
        ensure_device(c);
        if (!term_off || !term_f1 || !term_f2 || !annot || !directional || !directed ||
            K <= 0 || B <= 0 || F <= 0 || P <= 0 || variant_block <= 0 || !(residual_rank > 0.0))
            fail(LDS_ERR_ARG, "invalid generalized pass-2 arguments");
        const int cols = K * B * F;
        if (gen_rows_smem_bytes(cols) > (size_t)kGenRowsMaxSmem)
            fail(LDS_ERR_ARG, "K * B * families = %d right-hand-side columns exceeds %d", cols,
                 (int)(kGenRowsMaxSmem / sizeof(double)));
        if (c.slices != 4 || p2_impl() != 1)
            fail(LDS_ERR_ARG, "generalized products need the tcgen05 kernels with 4 digits");
        const Prepared& img = product_image(geno, 0, 1, cols);
        const int64_t M = img.g.M, N = img.g.N, Np = img.g.N_pad;
        const int nterm = term_off[P * P];
        for (int t = 0; t < nterm; ++t)
            if (term_f1[t] < 0 || term_f1[t] >= F || term_f2[t] < 0 || term_f2[t] >= F)
                fail(LDS_ERR_ARG, "orientation term family out of range");
        // The right-hand side as K2 bins of 64 columns (zero columns pad the
        // last), quantized to the phase-2 digits once for every block.
        constexpr int kV2 = 64;
        const int K2 = (cols + kV2 - 1) / kV2, nc = umma::ncolp_for(kV2);
        const int64_t ld = (int64_t)K2 * kV2;
        DevBuf dY, dyq, dcs, dann, dto, df1, df2, ddir, drg, dro, drows, dst;
        double* Y = dY.as<double>((size_t)(Np * ld));
        ck(cudaMemsetAsync(Y, 0, sizeof(double) * (size_t)(Np * ld), c.st), "memset");
        fill(Y, N, Np);
        int8_t* yq = dyq.as<int8_t>((size_t)((int64_t)K2 * nc * Np));
        double* cs = dcs.as<double>((size_t)ld);
        umma::launch_quantize_y4(Y, N, Np, K2, kV2, nc, yq, cs, c.st);
        double* ann = dann.as<double>((size_t)(M * K));
        h2d(ann, annot, (size_t)(M * K), c.st);
        int* to = dto.as<int>((size_t)(P * P + 1));
        int* f1 = df1.as<int>((size_t)std::max(nterm, 1));
        int* f2 = df2.as<int>((size_t)std::max(nterm, 1));
        h2d(to, term_off, (size_t)(P * P + 1), c.st);
        h2d(f1, term_f1, (size_t)nterm, c.st);
        h2d(f2, term_f2, (size_t)nterm, c.st);
        const int Cc = K * P;
        double* dd = ddir.as<double>((size_t)(Cc * Cc));
        ck(cudaMemsetAsync(dd, 0, sizeof(double) * (size_t)(Cc * Cc), c.st), "memset");
        unsigned* stv = dst.as<unsigned>(1);
        ck(cudaMemsetAsync(stv, 0, 4, c.st), "memset");
        const int64_t Lmax = std::min<int64_t>(variant_block, M);
        long long* rg = drg.as<long long>((size_t)(Lmax * ld));
        long long* ro = dro.as<long long>((size_t)(Lmax * ld));
        double* rows = drows.as<double>((size_t)(Lmax * P * Cc));
        const CUtensorMap tA = make_map_2d(img.g.codes, (uint64_t)img.g.nbp, (uint64_t)img.g.M_pad,
                                           (uint64_t)img.g.nbp, 32, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
        for (int64_t j0 = 0; j0 < M; j0 += Lmax) {
            const int64_t j1 = std::min(M, j0 + Lmax), L = j1 - j0;
            umma::P2UArgs u;
            u.yq = yq;
            u.yq_cols = (int64_t)K2 * nc;
            u.K = K2;
            u.V = kV2;
            u.ncolp = nc;
            u.bins_per_cta = umma::p2_bins_per_cta(nc, K2);
            u.ngroups = (u.bins_per_cta * nc + 255) / 256;
            u.box_rows = std::min(256, u.bins_per_cta * nc);
            u.nkt = (int)(Np / 128);
            u.M = M;
            u.j0 = j0;
            u.j1 = j1;
            u.out_row0 = j0;
            u.colscale = cs;
            u.mean = static_cast<double*>(img.d_mean.p);
            u.sdinv = static_cast<double*>(img.d_sdinv.p);
            u.status = stv;
            u.raw_g = rg;
            u.raw_o = ro;
            umma::launch_p2_umma(tA, u, c.st);
            launch_gen_rows(rg, ro, ld, cs, static_cast<double*>(img.d_mean.p),
                            static_cast<double*>(img.d_sdinv.p), j0, L, 1.0 / residual_rank, K, B, F,
                            P, to, f1, f2, rows, c.st);
            launch_gen_directed(rows, L, ann, j0, K, P, dd, c.st);
            ck(cudaGetLastError(), "launch");
            d2h(directional + j0 * P * Cc, rows, (size_t)(L * P * Cc), c.st);
        }
        unsigned hst = 0;
        d2h(directed, dd, (size_t)(Cc * Cc), c.st);
        d2h(&hst, stv, 1, c.st);
        ck(cudaStreamSynchronize(c.st), "generalized pass 2");
        if (hst) fail(LDS_ERR_CUDA, "phase-2 tensor-core pipeline wait timed out (code %u)", hst);
    }
}

LDS_API int lds_generalized_pass2(int64_t geno, const double* rhs, int K, int B, int F, int P,
                                  const int* term_off, const int* term_f1, const int* term_f2,
                                  double residual_rank, const double* annot,
                                  int64_t variant_block, double* directional, double* directed) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!rhs) fail(LDS_ERR_ARG, "invalid generalized pass-2 arguments");
        const int cols = K * B * F;
        gen_pass2_run(
            c, geno,
            [&](double* Y, int64_t N, int64_t Np) {
                ck(cudaMemcpy2DAsync(Y, sizeof(double) * (size_t)Np, rhs, sizeof(double) * (size_t)N,
                                     sizeof(double) * (size_t)N, (size_t)cols,
                                     cudaMemcpyHostToDevice, c.st),
                   "rhs upload");
            },
            K, B, F, P, term_off, term_f1, term_f2, residual_rank, annot, variant_block,
            directional, directed);
    });
}

LDS_API int lds_generalized_project(const double* base, const double* basis, const double* fixed,
                                    int K, int Q, int B, int R, int64_t N, double* contextual,
                                    double* max_abs, double* max_rel) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        if (!base || !basis || (R > 0 && !fixed) || !contextual || K <= 0 || Q <= 0 || B <= 0 ||
            R < 0 || R > kGenMaxR || N <= 0)
            fail(LDS_ERR_ARG, "invalid generalized projection arguments");
        const int64_t rows = (int64_t)K * Q * B;
        DevBuf dbase, dbasis, dfixed, dout, dleak, dpn;
        double* db = dbase.as<double>((size_t)((int64_t)K * B * N));
        h2d(db, base, (size_t)((int64_t)K * B * N), c.st);
        double* dq = dbasis.as<double>((size_t)(N * Q));
        h2d(dq, basis, (size_t)(N * Q), c.st);
        double* df = nullptr;
        if (R > 0) {
            df = dfixed.as<double>((size_t)(N * R));
            h2d(df, fixed, (size_t)(N * R), c.st);
        }
        double* o = dout.as<double>((size_t)(rows * N));
        double* lk2 = dleak.as<double>((size_t)std::max<int64_t>(rows * R, 1));
        double* pn = dpn.as<double>((size_t)rows);
        launch_gen_project(db, dq, Q, df, R, K, B, N, o, lk2, pn, c.st);
        ck(cudaGetLastError(), "launch");
        std::vector<double> hl((size_t)(rows * R)), hp((size_t)rows);
        d2h(contextual, o, (size_t)(rows * N), c.st);
        if (R > 0) d2h(hl.data(), lk2, hl.size(), c.st);
        d2h(hp.data(), pn, hp.size(), c.st);
        ck(cudaStreamSynchronize(c.st), "generalized projection");
        // the reference's leakage measures: the largest |fixed^T p| entry, and
        // per (k, q) ||fixed^T P||_F / max(1, ||P||_F); zero without fixed effects
        double mabs = 0.0, mrel = 0.0;
        if (R > 0)
            for (int64_t kq = 0; kq < (int64_t)K * Q; ++kq) {
                double l2 = 0.0, p2 = 0.0;
                for (int b = 0; b < B; ++b) {
                    const int64_t row = kq * B + b;
                    p2 += hp[(size_t)row];
                    for (int r = 0; r < R; ++r) {
                        const double v = hl[(size_t)(row * R + r)];
                        mabs = std::max(mabs, std::fabs(v));
                        l2 += v * v;
                    }
                }
                mrel = std::max(mrel, std::sqrt(l2) / std::max(1.0, std::sqrt(p2)));
            }
        if (max_abs) *max_abs = mabs;
        if (max_rel) *max_rel = mrel;
    });
}

LDS_API int lds_generalized_pass2_sources(int64_t geno, const double* sources, int Q,
                                          const double* basis, const int* fam_t,
                                          const int* fam_s, int K, int B, int F, int P,
                                          const int* term_off, const int* term_f1,
                                          const int* term_f2, double residual_rank,
                                          const double* annot, int64_t variant_block,
                                          double* directional, double* directed) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!sources || !basis || !fam_t || !fam_s || Q <= 0 || F <= 0)
            fail(LDS_ERR_ARG, "invalid generalized pass-2 arguments");
        for (int f = 0; f < F; ++f)
            if (fam_t[f] < 0 || fam_t[f] >= Q || fam_s[f] < 0 || fam_s[f] >= Q)
                fail(LDS_ERR_ARG, "family basis index out of range");
        DevBuf dS, dbasis, dft, dfs;
        gen_pass2_run(
            c, geno,
            [&](double* Y, int64_t N, int64_t Np) {
                // the sources (K Q B rows of N samples) and the basis cross
                // PCIe; the K B F family columns are formed on the device
                const int64_t rows = (int64_t)K * Q * B;
                double* S = dS.as<double>((size_t)(rows * Np));
                ck(cudaMemcpy2DAsync(S, sizeof(double) * (size_t)Np, sources,
                                     sizeof(double) * (size_t)N, sizeof(double) * (size_t)N,
                                     (size_t)rows, cudaMemcpyHostToDevice, c.st),
                   "sources upload");
                double* bs = dbasis.as<double>((size_t)(N * Q));
                h2d(bs, basis, (size_t)(N * Q), c.st);
                int* ft = dft.as<int>((size_t)F);
                int* fs = dfs.as<int>((size_t)F);
                h2d(ft, fam_t, (size_t)F, c.st);
                h2d(fs, fam_s, (size_t)F, c.st);
                launch_gen_assemble_rhs(S, Np, bs, Q, ft, fs, K, B, F, N, Y, c.st);
            },
            K, B, F, P, term_off, term_f1, term_f2, residual_rank, annot, variant_block,
            directional, directed);
    });
}

LDS_API int lds_gxe_destroy(int64_t gxe) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.ready) ck(cudaStreamSynchronize(c.st), "sync");
        gxe_table().erase(gxe);
    });
}

LDS_API int lds_gxe_set_checks(int64_t gxe, int on) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        GxeCtx& g = gxe_of(gxe);
        if (on && !g.P) fail(LDS_ERR_ARG, "product checks need a resident genotype image");
        g.check = on ? 1 : 0;
        g.chk_rows = g.chk_bad = 0;
        g.chk_first = -1;
    });
}

LDS_API int lds_gxe_last_check(int64_t gxe, unsigned long long* lhs, unsigned long long* rhs,
                               int64_t* first_row, int64_t* rows, int64_t* mismatches,
                               int64_t* first_snp) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        const GxeCtx& g = gxe_of(gxe);
        if (!g.check) fail(LDS_ERR_ARG, "product checks are off for this context (lds_gxe_set_checks)");
        if (lhs && g.chk_rows)
            std::memcpy(lhs, g.chk_hl.data(), sizeof(unsigned long long) * 2 * (size_t)g.chk_rows);
        if (rhs && g.chk_rows)
            std::memcpy(rhs, g.chk_hr.data(), sizeof(unsigned long long) * 2 * (size_t)g.chk_rows);
        if (first_row) *first_row = g.chk_j0;
        if (rows) *rows = g.chk_rows;
        if (mismatches) *mismatches = g.chk_bad;
        if (first_snp) *first_snp = g.chk_first;
    });
}

LDS_API int lds_gxe_source_block(int64_t gxe, int64_t j0, int64_t j1, const double* probes,
                                 int64_t B, const double* annotation, int annotation_is_sqrt,
                                 const double* scale_x, const double* scale_w, int64_t T,
                                 int environment_start, double* target, int device_ptrs) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!probes || !annotation || !scale_x || !scale_w || !target) fail(LDS_ERR_ARG, "null argument");
        gxe_source_impl(c, gxe_of(gxe), j0, j1, probes, B, annotation, annotation_is_sqrt, scale_x,
                        scale_w, T, environment_start, target, device_ptrs);
    });
}

LDS_API int lds_gxe_source_block_dense(int64_t gxe, const double* genotype, int64_t L,
                                       const double* probes, int64_t B, const double* annotation,
                                       int annotation_is_sqrt, const double* scale_x,
                                       const double* scale_w, int64_t T, int environment_start,
                                       double* target, int device_ptrs) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!genotype || !probes || !annotation || !scale_x || !scale_w || !target)
            fail(LDS_ERR_ARG, "null argument");
        gxe_source_impl(c, gxe_of(gxe), 0, L, probes, B, annotation, annotation_is_sqrt, scale_x,
                        scale_w, T, environment_start, target, device_ptrs, genotype);
    });
}

LDS_API int lds_gxe_target_score_block_dense(int64_t gxe, const double* genotype, int64_t L,
                                             int64_t pair, const double* scale_x,
                                             const double* scale_w, int64_t T, double* accum_xx,
                                             double* accum_xw, double* accum_wx, double* accum_ww,
                                             int64_t block_start, int64_t total_variants,
                                             int probe_count, int environment_start,
                                             int device_ptrs) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!genotype || !scale_x || !scale_w || !accum_xx || !accum_xw || !accum_wx || !accum_ww)
            fail(LDS_ERR_ARG, "null argument");
        gxe_target_impl(c, gxe_of(gxe), 0, L, gxe_pair_of(pair), scale_x, scale_w, T, accum_xx,
                        accum_xw, accum_wx, accum_ww, block_start, total_variants, probe_count,
                        environment_start, device_ptrs, genotype);
    });
}

LDS_API int lds_gxe_project_sources(int64_t gxe, double* panel, int64_t columns,
                                    int columns_per_environment, int environment_start,
                                    double* leakages, int device_ptrs) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!panel) fail(LDS_ERR_ARG, "null argument");
        gxe_project_impl(c, gxe_of(gxe), panel, columns, columns_per_environment, environment_start,
                         device_ptrs, leakages);
    });
}

LDS_API int lds_gxe_pair_create(int64_t gxe, const double* right, int64_t columns,
                                const double* row_weights, int64_t groups, int device_ptrs,
                                int64_t* pair_out) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!right || !row_weights) fail(LDS_ERR_ARG, "null argument");
        GxeCtx& g = gxe_of(gxe);
        auto pr = gxe_pair_impl(c, g, right, g.N, columns, row_weights, groups, device_ptrs);
        const int64_t h = next_handle();
        gxe_pair_table()[h] = std::move(pr);
        *pair_out = h;
    });
}

LDS_API int lds_gxe_pair_destroy(int64_t pair) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.ready) ck(cudaStreamSynchronize(c.st), "sync");
        gxe_pair_table().erase(pair);
    });
}

LDS_API int lds_gxe_target_score_block(int64_t gxe, int64_t j0, int64_t j1, int64_t pair,
                                       const double* scale_x, const double* scale_w, int64_t T,
                                       double* accum_xx, double* accum_xw, double* accum_wx,
                                       double* accum_ww, int64_t block_start, int64_t total_variants,
                                       int probe_count, int environment_start, int device_ptrs) {
    return guarded([&] {
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        if (!scale_x || !scale_w || !accum_xx || !accum_xw || !accum_wx || !accum_ww)
            fail(LDS_ERR_ARG, "null argument");
        gxe_target_impl(c, gxe_of(gxe), j0, j1, gxe_pair_of(pair), scale_x, scale_w, T, accum_xx,
                        accum_xw, accum_wx, accum_ww, block_start, total_variants, probe_count,
                        environment_start, device_ptrs);
    });
}

LDS_API int lds_gxe_normalize_scores(double* accum_xx, double* accum_xw, double* accum_wx,
                                     double* accum_ww, int64_t rows, int64_t K, int probe_count,
                                     int device_ptrs) {
    return guarded([&] {
        if (probe_count <= 0)
            fail(LDS_ERR_ARG, "Multi-environment native score normalization requires probes");
        if (rows <= 0 || K <= 0) fail(LDS_ERR_ARG, "Multi-environment native score normalization shape is invalid");
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        const size_t n = (size_t)(rows * K);
        double* hs[4] = {accum_xx, accum_xw, accum_wx, accum_ww};
        DevBuf tmp;
        double* base = device_ptrs ? nullptr : tmp.as<double>(4 * n);
        for (int q = 0; q < 4; ++q) {
            double* d = device_ptrs ? hs[q] : base + (size_t)q * n;
            if (!device_ptrs) h2d(d, hs[q], n, c.st);
            launch_scale(d, (int64_t)n, 1.0 / (double)probe_count, c.st);
        }
        // non-finite check (gxeldcore.cpp:12540-12550)
        DevBuf fl;
        unsigned* flag = fl.as<unsigned>(1);
        ck(cudaMemsetAsync(flag, 0, 4, c.st), "memset");
        for (int q = 0; q < 4; ++q) {
            double* d = device_ptrs ? hs[q] : base + (size_t)q * n;
            launch_gxe_check(d, (int64_t)n, d, d, 0, d, 0, flag, c.st);
            if (!device_ptrs) d2h(hs[q], d, n, c.st);
        }
        unsigned fv = 0;
        d2h(&fv, flag, 1, c.st);
        ck(cudaStreamSynchronize(c.st), "normalize");
        if (fv) fail(LDS_ERR_ARG, "Multi-environment native normalized scores are non-finite");
    });
}

LDS_API int lds_philox_rademacher(const uint64_t* keys, int64_t probes, int64_t rows, double* out,
                                  int device_ptrs) {
    return guarded([&] {
        if (!keys || !out || rows <= 0 || probes <= 0)
            fail(LDS_ERR_ARG, "Native Philox Rademacher inputs are invalid");
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        DevBuf k, o;
        const uint64_t* dk = keys;
        double* dout = out;
        if (!device_ptrs) {
            uint64_t* kk = k.as<uint64_t>((size_t)(2 * probes));
            h2d(kk, keys, (size_t)(2 * probes), c.st);
            dk = kk;
            dout = o.as<double>((size_t)(rows * probes));
        }
        launch_philox_rademacher(dk, probes, rows, dout, c.st);
        ck(cudaGetLastError(), "launch");
        if (!device_ptrs) d2h(out, dout, (size_t)(rows * probes), c.st);
        ck(cudaStreamSynchronize(c.st), "philox");
    });
}


// ---------------------------------------------------------------------------
// SNP-block jackknife and normal-equation solves (include/lds.h)
// ---------------------------------------------------------------------------
namespace {
// NumPy's pairwise summation of float64 (the algorithm behind np.sum): blocks
// of 8 partial sums up to 128 elements, halves (rounded to a multiple of 8)
// above that.
double pairwise_sum(const double* a, int64_t n) {
    if (n < 8) {
        double r = 0.0;
        for (int64_t i = 0; i < n; ++i) r += a[i];
        return r;
    }
    if (n <= 128) {
        double r[8];
        for (int k = 0; k < 8; ++k) r[k] = a[k];
        int64_t i = 8;
        for (; i < n - (n % 8); i += 8)
            for (int k = 0; k < 8; ++k) r[k] += a[i + k];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += a[i];
        return res;
    }
    int64_t n2 = n / 2;
    n2 -= n2 % 8;
    return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
}
}  // namespace

LDS_API int lds_block_boundaries(int64_t M, int B, const double* mass, int min_snps,
                                 int64_t* starts, int64_t* ends) {
    return guarded([&] {
        if (!(1 <= B && B <= M)) fail(LDS_ERR_ARG, "Need 1 <= nblocks <= nsnps, got B=%d, M=%lld", B, (long long)M);
        auto equal = [&] {
            // edges = floor(linspace(0, M, B + 1)), last edge M (jackknife.py:109-118)
            const double step = (double)M / (double)B;
            std::vector<int64_t> e((size_t)B + 1);
            for (int i = 0; i < B; ++i) e[(size_t)i] = (int64_t)std::floor((double)i * step);
            e[(size_t)B] = M;
            for (int i = 0; i < B; ++i) {
                starts[i] = e[(size_t)i];
                ends[i] = e[(size_t)i + 1];
                if (ends[i] <= starts[i]) fail(LDS_ERR_INTERNAL, "Equal-count partition produced an empty block.");
            }
        };
        if (!mass) {
            equal();
            return;
        }
        // weighted contiguous boundaries (jackknife.py:156-211)
        if (min_snps <= 0) fail(LDS_ERR_ARG, "min_snps must be >= 1");
        if ((int64_t)min_snps * B > M)
            fail(LDS_ERR_ARG, "min_snps * nblocks exceeds nsnps: %d * %d > %lld", min_snps, B, (long long)M);
        std::vector<double> m((size_t)M);
        for (int64_t j = 0; j < M; ++j)
            m[(size_t)j] = (std::isfinite(mass[j]) && mass[j] > 0.0) ? mass[j] : 0.0;
        const double total = pairwise_sum(m.data(), M);
        if (!(std::isfinite(total) && total > 0.0)) {
            equal();
            return;
        }
        std::vector<double> cs((size_t)M);
        double acc = 0.0;
        for (int64_t j = 0; j < M; ++j) cs[(size_t)j] = (acc += m[(size_t)j]);
        int64_t st = 0;
        for (int b = 0; b < B; ++b) {
            starts[b] = st;
            const int rem = B - b - 1;
            int64_t e;
            if (rem == 0) {
                e = M;
            } else {
                const int64_t low = st + min_snps, high = M - (int64_t)rem * min_snps;
                const double target = (double)(b + 1) * total / (double)B;
                e = (int64_t)(std::lower_bound(cs.begin(), cs.end(), target) - cs.begin()) + 1;
                if (e < low) e = low;
                if (e > high) e = high;
            }
            ends[b] = e;
            st = e;
        }
        if (starts[0] != 0 || ends[B - 1] != M)
            fail(LDS_ERR_INTERNAL, "Weighted contiguous partition produced invalid block boundaries.");
        for (int b = 0; b < B; ++b)
            if (ends[b] <= starts[b])
                fail(LDS_ERR_INTERNAL, "Weighted contiguous partition produced invalid block boundaries.");
    });
}

// Systems laid out as nsys x (K*K row-major matrix, K rhs).
static void sym_solve_impl(Context& c, const double* dsys, int64_t nsys, int K, double rtol,
                           int require_full_rank, double* x, int* rank, double* eig,
                           int device_ptrs) {
    if (K <= 0 || K > sym_solve_max_k()) fail(LDS_ERR_ARG, "system size must be in [1, %d]", sym_solve_max_k());
    if (!std::isfinite(rtol) || rtol <= 0.0) fail(LDS_ERR_ARG, "rtol must be finite and positive.");
    DevBuf dx, dr, de, dstat;
    // The kernel writes x, rank and eigenvalues of every system: each gets a
    // device buffer of its own unless the caller passed a device pointer.
    double* xo = (device_ptrs && x) ? x : dx.as<double>((size_t)(nsys * K));
    int* ro = (device_ptrs && rank) ? rank : dr.as<int>((size_t)nsys);
    double* eo = (device_ptrs && eig) ? eig : de.as<double>((size_t)(nsys * K));
    int* so = dstat.as<int>((size_t)nsys);
    launch_sym_solve(dsys, nsys, K, rtol, require_full_rank, xo, ro, eo, so, c.st);
    ck(cudaGetLastError(), "launch");
    std::vector<int> st((size_t)nsys), rk((size_t)nsys);
    d2h(st.data(), so, st.size(), c.st);
    d2h(rk.data(), ro, rk.size(), c.st);
    if (!device_ptrs) {
        if (x) d2h(x, xo, (size_t)(nsys * K), c.st);
        if (rank) d2h(rank, ro, (size_t)nsys, c.st);
        if (eig) d2h(eig, eo, (size_t)(nsys * K), c.st);
    }
    ck(cudaStreamSynchronize(c.st), "solve");
    for (int64_t q = 0; q < nsys; ++q) {
        if (st[(size_t)q] & 4) fail(LDS_ERR_ARG, "normal matrix contains non-finite values.");
        if (st[(size_t)q] & 1) fail(LDS_ERR_ARG, "Normal matrix has material asymmetry.");
        if (st[(size_t)q] & 2)
            fail(LDS_ERR_ARG, "Contextual normal system is not identifiable: rank %d of %d.",
                 rk[(size_t)q], K);
    }
}

LDS_API int lds_sym_solve(const double* systems, int64_t nsys, int K, double rtol,
                          int require_full_rank, double* x, int* rank, double* eigenvalues,
                          int device_ptrs) {
    return guarded([&] {
        if (!systems || nsys <= 0) fail(LDS_ERR_ARG, "no systems");
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        DevBuf ds;
        const double* d = systems;
        if (!device_ptrs) {
            double* t = ds.as<double>((size_t)(nsys * (K * K + K)));
            h2d(t, systems, (size_t)(nsys * (K * K + K)), c.st);
            d = t;
        }
        sym_solve_impl(c, d, nsys, K, rtol, require_full_rank, x, rank, eigenvalues, device_ptrs);
    });
}

LDS_API int lds_sym_solve_diag(const double* systems, int64_t nsys, int K, double rtol,
                               double* x, int* rank, double* eigenvalues, double* eigenvectors,
                               double* residual, double* symmetry_error, double* tolerance,
                               int* status) {
    return guarded([&] {
        if (!systems || nsys <= 0) fail(LDS_ERR_ARG, "no systems");
        if (K <= 0 || K > sym_solve_max_k())
            fail(LDS_ERR_ARG, "system size must be in [1, %d]", sym_solve_max_k());
        if (!std::isfinite(rtol) || rtol <= 0.0) fail(LDS_ERR_ARG, "rtol must be finite and positive.");
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        const size_t n = (size_t)nsys, k = (size_t)K;
        DevBuf ds, dx, dr, de, dv, dres, da, dt, dst;
        double* d = ds.as<double>(n * (k * k + k));
        h2d(d, systems, n * (k * k + k), c.st);
        SymSolveExtras ex;
        ex.evec = dv.as<double>(n * k * k);
        ex.resid = dres.as<double>(n * k);
        ex.asym = da.as<double>(n);
        ex.tol = dt.as<double>(n);
        double* xo = dx.as<double>(n * k);
        int* ro = dr.as<int>(n);
        double* eo = de.as<double>(n * k);
        int* so = dst.as<int>(n);
        launch_sym_solve(d, nsys, K, rtol, 0, xo, ro, eo, so, c.st, ex);
        ck(cudaGetLastError(), "launch");
        if (x) d2h(x, xo, n * k, c.st);
        if (rank) d2h(rank, ro, n, c.st);
        if (eigenvalues) d2h(eigenvalues, eo, n * k, c.st);
        if (eigenvectors) d2h(eigenvectors, ex.evec, n * k * k, c.st);
        if (residual) d2h(residual, ex.resid, n * k, c.st);
        if (symmetry_error) d2h(symmetry_error, ex.asym, n, c.st);
        if (tolerance) d2h(tolerance, ex.tol, n, c.st);
        if (status) d2h(status, so, n, c.st);
        ck(cudaStreamSynchronize(c.st), "solve");
    });
}

LDS_API int lds_jackknife_normal_equations(const double* terms, int64_t M, int K,
                                           const int64_t* starts, const int64_t* ends, int64_t B,
                                           double rtol, double* theta, double* replicates,
                                           double* se, double* cov, int device_ptrs) {
    return guarded([&] {
        if (!terms || !starts || !ends || M <= 0 || B <= 1) fail(LDS_ERR_ARG, "invalid jackknife inputs");
        for (int64_t b = 0; b < B; ++b)
            if (starts[b] < 0 || ends[b] > M || ends[b] <= starts[b])
                fail(LDS_ERR_ARG, "invalid jackknife block boundaries");
        Context& c = ctx();
        std::lock_guard<std::mutex> lk(c.mu);
        ensure_device(c);
        const int64_t P = (int64_t)K * K + K;
        DevBuf dt, dst, den, dblk, dsys, dx, dr, de, dmean, dse, dcov;
        const double* t = terms;
        if (!device_ptrs) {
            double* p = dt.as<double>((size_t)(M * P));
            h2d(p, terms, (size_t)(M * P), c.st);
            t = p;
        }
        int64_t* s_ = dst.as<int64_t>((size_t)B);
        int64_t* e_ = den.as<int64_t>((size_t)B);
        h2d(s_, starts, (size_t)B, c.st);
        h2d(e_, ends, (size_t)B, c.st);
        double* blk = dblk.as<double>((size_t)(B * P));
        launch_block_sums(t, P, s_, e_, B, blk, c.st);
        double* sys = dsys.as<double>((size_t)((B + 1) * P));
        launch_delete_one(blk, B, P, sys, c.st);
        double* xs = dx.as<double>((size_t)((B + 1) * K));
        sym_solve_impl(c, sys, B + 1, K, rtol, 0, xs, nullptr, nullptr, 1);
        double* mean = dmean.as<double>((size_t)K);
        double* sed = dse.as<double>((size_t)K);
        double* cv = dcov.as<double>((size_t)(K * K));
        launch_jackknife_stats(xs + K, B, K, mean, sed, cv, c.st);
        ck(cudaGetLastError(), "launch");
        auto out = [&](double* dst_, const double* src, size_t n) {
            if (!dst_) return;
            if (device_ptrs) ck(cudaMemcpyAsync(dst_, src, n * sizeof(double), cudaMemcpyDeviceToDevice, c.st), "copy");
            else d2h(dst_, src, n, c.st);
        };
        out(theta, xs, (size_t)K);
        out(replicates, xs + K, (size_t)(B * K));
        out(se, sed, (size_t)K);
        out(cov, cv, (size_t)(K * K));
        ck(cudaStreamSynchronize(c.st), "jackknife");
    });
}
