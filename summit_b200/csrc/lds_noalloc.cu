// Phase 2 for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc while they run this step: code running
// inside a CUDA stream capture (allocation breaks the capture), programs whose
// device memory belongs to another framework's pool, and long-running services
// that forbid allocator calls after start-up because those calls synchronize
// the device or fragment memory.  They own their input and output buffers but
// need the library to bring its own scratch.  This entry point keeps its
// scratch — the 4-digit int8 split of the sketch, the per-column scales, a
// status word and two guard counters — in one file-scope __device__ array of
// fixed size (kNoallocScratchBytes, 16 MiB).  Every GPU that loads the library
// holds that array until the process exits.
//
// Rules of use:
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current).  Make
//     that first call before any stream capture that includes this entry.
//   * All calls share the one array, and it keeps the last call's contents.
//     Calls whose work can overlap on the GPU (different streams, or host
//     threads without ordering) race on it; serialize them.
//   * Sizes that do not fit are rejected with LDS_ERR_ARG and a message giving
//     the bytes needed and the limit; nothing is allocated.
//   * The kernel's status word (nonzero when a pipeline wait ran out) and its
//     guard counters (non-finite / extreme updates dropped) are copied on the
//     same stream into caller-owned device words when the caller passes them,
//     so the call stays asynchronous.  Without them the call waits for its own
//     work on the stream and returns the status itself, so a failed kernel is
//     never reported as LDS_OK.
// It calls no cudaMalloc, cudaFree or allocating library routine.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <cudaTypedefs.h>

#include "../../include/lds.h"
#include "lds_internal.h"
#include "lds_umma.h"

namespace lds {
namespace noalloc {

constexpr size_t kNoallocScratchBytes = LDS_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeaderBytes = 256;  // status word + guard counters, then column scales

static __device__ __align__(256) uint8_t g_scratch[kNoallocScratchBytes];

// Error text goes to the library's lds_last_error().
struct Msg {
    Msg& operator=(const std::string& m) {
        set_last_error(m);
        return *this;
    }
    Msg& operator=(const char* m) { return *this = std::string(m); }
};
static Msg g_msg;

struct DevSlot {
    bool ready = false;
    uint8_t* addr = nullptr;
};

// Device address of g_scratch for the current device (looked up once per device).
static int scratch_address(uint8_t** out) {
    static std::mutex mu;
    static DevSlot slots[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        g_msg = "no current CUDA device";
        return LDS_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!slots[dev].ready) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            g_msg = std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                    cudaGetErrorString(e);
            return LDS_ERR_CUDA;
        }
        // The phase-2 kernel's shared-memory limit is a per-device attribute;
        // set it here too, so that it is in place before any capture.
        umma::prepare_p2_umma();
        slots[dev].addr = static_cast<uint8_t*>(p);
        slots[dev].ready = true;
    }
    *out = slots[dev].addr;
    return LDS_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

static bool map2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint64_t stride,
                  uint32_t bi, uint32_t bo, CUtensorMapSwizzle swz) {
    auto enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {stride};
    const cuuint32_t box[2] = {bi, bo};
    const cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int run(const uint8_t* d_codes, int64_t row_bytes, int64_t n, int64_t rows_total,
               int64_t j0, int64_t j1, const double* d_Y, int K, int V, const double* d_mean,
               const double* d_sdinv, const double* d_left_scale, double* d_accum, double* d_mc,
               unsigned* d_status_out, unsigned long long* d_guards_out, cudaStream_t st) {
    if (!d_codes || !d_Y || !d_mean || !d_sdinv || !d_left_scale || !d_accum) {
        g_msg = "null device pointer";
        return LDS_ERR_ARG;
    }
    if (row_bytes <= 0 || row_bytes % 64 != 0) {
        g_msg = "row_bytes must be a positive multiple of 64 (samples padded to 256)";
        return LDS_ERR_ARG;
    }
    const int64_t N_pad = row_bytes * 4;
    if (n <= 0 || n > N_pad || K <= 0 || V <= 0 || j0 < 0 || j1 <= j0 || rows_total < j1) {
        g_msg = "invalid sizes (need 0 < n <= 4*row_bytes, K > 0, V > 0, 0 <= j0 < j1 <= rows_total)";
        return LDS_ERR_ARG;
    }
    if ((reinterpret_cast<uintptr_t>(d_codes) & 15) != 0) {
        g_msg = "d_codes must be 16-byte aligned";
        return LDS_ERR_ARG;
    }
    const int ncolp = umma::ncolp_for(V);
    const size_t digits = (size_t)K * (size_t)ncolp * (size_t)N_pad;
    const size_t need = kHeaderBytes + ((sizeof(double) * (size_t)K * V + 1023) / 1024) * 1024 + digits;
    if (need > kNoallocScratchBytes) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "sizes need %zu bytes of scratch; the no-allocation entry has %zu "
                      "(K * ceil16(4 V) * N_pad digit bytes must stay under it)",
                      need, kNoallocScratchBytes);
        g_msg = buf;
        return LDS_ERR_ARG;
    }
    uint8_t* scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    unsigned* status = reinterpret_cast<unsigned*>(scratch);
    unsigned long long* guards = reinterpret_cast<unsigned long long*>(scratch + 64);
    double* colscale = reinterpret_cast<double*>(scratch + kHeaderBytes);
    int8_t* yq = reinterpret_cast<int8_t*>(
        scratch + kHeaderBytes + ((sizeof(double) * (size_t)K * V + 1023) / 1024) * 1024);

    // The status word and guard counters must start at zero for this call.
    if (cudaMemsetAsync(scratch, 0, 128, st) != cudaSuccess) {
        g_msg = "cudaMemsetAsync of the status words failed";
        return LDS_ERR_CUDA;
    }
    CUtensorMap tA;
    if (!map2d(&tA, d_codes, (uint64_t)row_bytes, (uint64_t)rows_total, (uint64_t)row_bytes, 32, 128,
               CU_TENSOR_MAP_SWIZZLE_NONE)) {
        g_msg = "cuTensorMapEncodeTiled failed";
        return LDS_ERR_CUDA;
    }
    umma::launch_quantize_y4(d_Y, n, N_pad, K, V, ncolp, yq, colscale, st);
    umma::P2UArgs u;
    u.K = K;
    u.V = V;
    u.ncolp = ncolp;
    u.ngroups = (ncolp + 255) / 256;
    u.box_rows = ncolp < 256 ? ncolp : 256;
    u.nkt = (int)(N_pad / 128);
    u.M = j1;  // per-SNP statistics are read for rows < j1 only
    u.j0 = j0;
    u.j1 = j1;
    u.out_row0 = j0;
    u.colscale = colscale;
    u.mean = d_mean;
    u.sdinv = d_sdinv;
    u.left_scale = d_left_scale;
    u.accum = d_accum;
    u.mc = d_mc;
    u.guard_counts = guards;
    u.extreme_warn = phase2_extreme_warn();
    u.drop_extreme = phase2_drop_extreme();
    u.status = status;
    u.yq = yq;
    u.yq_cols = (int64_t)K * ncolp;
    umma::launch_p2_umma(tA, u, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_msg = std::string("launch failed: ") + cudaGetErrorString(e);
        return LDS_ERR_CUDA;
    }
    if (d_status_out || d_guards_out) {
        // Asynchronous report: the header words follow the kernel on `st`.
        if (d_status_out)
            e = cudaMemcpyAsync(d_status_out, status, sizeof(unsigned), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && d_guards_out)
            e = cudaMemcpyAsync(d_guards_out, guards, 2 * sizeof(unsigned long long),
                                cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            g_msg = std::string("copy of the status words failed: ") + cudaGetErrorString(e);
            return LDS_ERR_CUDA;
        }
        return LDS_OK;
    }
    // No caller-owned status words: wait for this call's work and read them
    // here (into host stack memory; nothing is allocated).
    unsigned h_status = 0;
    unsigned long long h_guards[2] = {0, 0};
    e = cudaMemcpyAsync(&h_status, status, sizeof h_status, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_guards, guards, sizeof h_guards, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        g_msg = std::string("phase 2 failed: ") + cudaGetErrorString(e);
        return LDS_ERR_CUDA;
    }
    if (h_guards[0])
        std::fprintf(stderr,
                     "[phase2-warning] noalloc rows [%lld:%lld): dropped %llu non-finite LD-score "
                     "updates.\n",
                     (long long)j0, (long long)j1, h_guards[0]);
    if (h_guards[1])
        std::fprintf(stderr,
                     "[phase2-warning] noalloc rows [%lld:%lld): %llu finite updates exceeded the "
                     "LD-score warning threshold. They were %s; inspect this run before using it.\n",
                     (long long)j0, (long long)j1, h_guards[1],
                     u.drop_extreme ? "dropped" : "kept");
    if (h_status) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "phase-2 kernel aborted: a pipeline wait ran out (status %u); the "
                      "accumulators are incomplete",
                      h_status);
        g_msg = buf;
        return LDS_ERR_CUDA;
    }
    return LDS_OK;
}

}  // namespace noalloc
}  // namespace lds

extern "C" __attribute__((visibility("default"))) int lds_phase2_accum_device_noalloc(
    const uint8_t* d_codes, int64_t row_bytes, int64_t n, int64_t rows_total, int64_t j0,
    int64_t j1, const double* d_Y, int K, int V, const double* d_mean, const double* d_sdinv,
    const double* d_left_scale, double* d_accum, double* d_mc, unsigned* d_status,
    unsigned long long* d_guards, void* stream) {
    return lds::noalloc::run(d_codes, row_bytes, n, rows_total, j0, j1, d_Y, K, V, d_mean, d_sdinv,
                             d_left_scale, d_accum, d_mc, d_status, d_guards,
                             static_cast<cudaStream_t>(stream));
}

