// tcgen05 (UMMA) phase-2 kernel interface.
#pragma once
#include <climits>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace lds {
namespace umma {

// Sketch digits in phase 2's operand layout.  Column 4 v + t of bin k is digit
// t of probe v (global column k * ncolp + 4 v + t of `cols` columns).  The
// samples come in chunks of 128 (one phase-2 K-step): chunk kt holds every
// column's 128-byte row, contiguously ([kt][cols][128 bytes]), and each
// 8-row group (1 KB) is pre-swizzled as the SWIZZLE_128B K-major UMMA atom
// expects (16-byte chunk index XOR row & 7).  A K-step's tile of any run of
// columns starting on a multiple of 8 is then one contiguous block that a
// single bulk copy moves into shared memory ready for the MMA.
__host__ __device__ inline int64_t digit_offset(int64_t col, int64_t i, int64_t cols) {
    const int s = (int)(i & 127);
    return ((i >> 7) * cols + col) * 128 + ((((s >> 4) ^ (int)(col & 7)) << 4) | (s & 15));
}

// Arguments of p2_umma_kernel.  The sketch digits are yq (digit_offset layout
// with yq_cols columns): per bin, ncolp columns.
struct P2UArgs {
    int K = 0, V = 0, ncolp = 0, ngroups = 1, box_rows = 0, nkt = 0;
    int64_t M = 0, j0 = 0, j1 = 0, out_row0 = 0;
    const double* colscale = nullptr;    // K*V
    const double* mean = nullptr;
    const double* sdinv = nullptr;
    const double* left_scale = nullptr;
    double* accum = nullptr;
    double* mc = nullptr;
    unsigned long long* guard_counts = nullptr;
    double extreme_warn = 1e10;
    int drop_extreme = 1;
    unsigned int* status = nullptr;      // 0 = ok; nonzero = pipeline wait timed out
    const int8_t* yq = nullptr;          // sketch digits (digit_offset layout)
    int64_t yq_cols = 0;                 // columns of yq (super-bins x ncolp)
    // Verification mode: write the exact recombined products G^T y and O^T y
    // per (SNP, bin, probe) to raw_g / raw_o (((j - out_row0) * K + k) * V + v),
    // no epilogue.
    long long* raw_g = nullptr;
    long long* raw_o = nullptr;
    // Optional tile table (windowed estimates): CTA x processes rows
    // [tiles[x].x, min(tiles[x].x + 128, tiles[x].y)) against super-bins
    // tiles[x].z + k (sketch columns and scales of that window).
    const int4* tiles = nullptr;
    // Optional split of the probes into two sums: probes v < split_v go to
    // accum, the rest to accum2 (guards judge their total).  Unused if null.
    double* accum2 = nullptr;
    int split_v = 0;
    // Bins per CTA (consecutive; one decoded genotype tile serves them all):
    // box_rows = min(256, bins_per_cta * ncolp) and ngroups =
    // ceil(bins_per_cta * ncolp / 256) must match.  1 unless ncolp <= 128.
    int bins_per_cta = 1;
    // Tiles with every call observed: snp_missing[j] != 0 marks SNP row j as
    // having a missing call.  A 128-SNP tile whose output rows have none
    // skips the O plane: its observed-count products O^T y equal the sketch
    // digits' column sums, colsum[global digit column] (int32, over all padded
    // samples; padding samples carry zero digits).  Unused if either is null.
    const uint8_t* snp_missing = nullptr;
    const int* colsum = nullptr;
    // Product checksums (lds_check.cu): when set, chk[2j] and chk[2j+1] gain
    // sum over this CTA's (bin k, probe v) of check_weight(k, chk_v0 + v) times
    // the exact products T_G and T_O of SNP row j (wrapping mod 2^64).
    unsigned long long* chk = nullptr;
    int chk_v0 = 0;
    // Optional CTA order: CTA x processes tile work[x].x (an entry of the tile
    // table, or rows j0 + 128 work[x].x without one) with bin group
    // work[x].y (n_work entries, the grid), instead of tile blockIdx.x and bin
    // group blockIdx.y.
    const int2* work = nullptr;
    int64_t n_work = 0;
    // Extent of accum / accum2 / mc in elements, read by the bounds-checked
    // build's output checks (0: unchecked).
    int64_t accum_elems = 0;
};

// Bins that share one CTA in phase 2: as many whole bins as fit 256 columns.
inline int p2_bins_per_cta(int ncolp, int K) {
    if (ncolp > 128) return 1;
    const int nb = 256 / ncolp;
    return nb < K ? nb : K;
}

// Bins per CTA for the plans that run phase 2 from a work order: the CTA
// walks its bins' columns in MMA groups of up to 256 (a bin may straddle two
// groups), so a tile costs ceil(K / nb) CTAs x ceil(nb * ncolp / 256) groups.
// The smallest nb with the fewest groups per tile: for 208-column bins and
// K = 24, nb = 6 (20 groups of 256 columns instead of 24 of 208; an MMA's
// cost is nearly the same at N = 208 and N = 256).
inline int p2_bins_per_cta_grouped(int ncolp, int K) {
    if (ncolp <= 128) return p2_bins_per_cta(ncolp, K);
    int best = 1;
    int64_t best_groups = INT64_MAX;
    for (int nb = 1; nb <= K; ++nb) {
        const int64_t groups =
            (int64_t)((K + nb - 1) / nb) * (((int64_t)nb * ncolp + 255) / 256);
        if (groups < best_groups) {
            best_groups = groups;
            best = nb;
        }
    }
    return best;
}

// Phase-1 tcgen05 kernel arguments.  Member lists of bin k occupy
// rowind[bin_off[k] .. bin_off[k+1]) (multiples of 128, padding rows carry
// zero weights); weight digits Wq[((k*2+part)*ncolp + 4v+t)*lmax + r].
struct P1UArgs {
    int K = 0, V = 0, ncolp = 0, ngroups = 1, box_rows = 0;
    int64_t nbp = 0, N_pad = 0;
    const int64_t* bin_off = nullptr;
    const int32_t* rowind = nullptr;
    const uint8_t* codes = nullptr;
    const double* colscale = nullptr;   // K*V
    double* Y = nullptr;                // N_pad x (K*V), column (k*V+v)
    unsigned int* status = nullptr;
    int sb_per_cta = 1;                 // super-bins processed by one CTA (pipeline continues)
    // Digit output (windowed estimates): when yq is set the epilogue writes the
    // sketch's 4 int8 digits in phase 2's layout (digit_offset, column
    // k*ncolp + 4v + t of K*ncolp) using the a-priori exponents in ycolscale
    // (K*V) instead of FP64 Y.
    int8_t* yq = nullptr;
    const double* ycolscale = nullptr;
    const int* yshift = nullptr;        // K*V digit shifts eW - eY (from the weight kernel)
    int64_t m_pad = 0;                  // image rows, for the bounds-checked build (0: unchecked)
};

struct P1UWeights {
    int K = 0, V = 0, ncolp = 0;
    int64_t lmax = 0;
    const int32_t* rowind = nullptr;
    const double* sc = nullptr;
    const int64_t* bin_off = nullptr;
    int8_t* wq = nullptr;
    double* colscale = nullptr;
    double* ycolscale = nullptr;        // optional: a-priori sketch digit scales (K*V)
    int* yshift = nullptr;              // with ycolscale: digit shifts eW - eY (K*V)
};

void launch_p1_weights4(const P1UWeights& w, const double* mean, const double* sdinv,
                        const double* Z, int64_t z_ld, cudaStream_t st);
size_t p1_umma_smem_bytes();
void launch_p1_umma(const CUtensorMap& tmW, const P1UArgs& a, int64_t N_pad, cudaStream_t st);

// Columns per bin (4 digits per probe, padded to a multiple of 16).
inline int ncolp_for(int V) { return ((4 * V + 15) / 16) * 16; }

// colsum (optional, K * ncolp ints): the digit columns' sums over all samples.
void launch_quantize_y4(const double* Y, int64_t N, int64_t N_pad, int K, int V, int ncolp,
                        int8_t* Yq, double* colscale, cudaStream_t st, int* colsum = nullptr);
// colsum[c] = sum over the N_pad samples of digit column c of Yq (ncols columns).
void launch_digit_colsum(const int8_t* Yq, int64_t ncols, int64_t N_pad, int* colsum,
                         cudaStream_t st);
size_t p2_umma_smem_bytes(int box_rows);
// Set the kernels' shared-memory attributes ahead of any stream capture.
void prepare_p2_umma();
void prepare_p1_umma();
void launch_p2_umma(const CUtensorMap& tmA, const P2UArgs& a, cudaStream_t st);

}  // namespace umma
}  // namespace lds
