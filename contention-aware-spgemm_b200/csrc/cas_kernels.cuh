// casgemm kernels for C = A * B on sm_100a (B = A^T in every benchmark
// configuration, but B is read as its own CSR, as in the reference).
//
// CSR layout in HBM: int64 row pointers, int32 column indices, values fp64
// (or int32 in / int64 out for the integer mode).  Every row of C is written
// with its columns sorted.
//
// Pipeline (the reference's four phases, src/ams_hybaccspgemm.c:36-215):
//   INIT  k_flp            row_flp[i] = sum_{k in A_i} |B_k|   (flp_populate,
//                          src/mm/mm_utils.c:1063-1125), total products
//         k_bin_*          rows binned by intermediate-product count: the
//                          GPU form of the morsel packing of pack_ams_pack
//                          (src/ams/ams_utils.c:1410-1596)
//   SYMB  k_symb_*         exact distinct-column count per row
//                          (ams_hash_symb_dnr, src/ams/ams_utils.c:1630-1752)
//         k_scan_*         exclusive scan -> C row pointers (scan,
//                          src/mm/mm_utils.c:866-957)
//   NUMC  k_numc_*         hash / ESC / hybrid accumulation
//                          (src/ams/ams_utils.c:168-475, 956-1338)
#pragma once
#include "cas_device.cuh"

namespace cas {

// ------------------------------------------------------------ parameters
// Symbolic bins by t = min(row_flp, num_col) (an upper bound on the row's
// distinct columns); numeric bins by accumulator and size.
// Hash tables hold at least twice the bound, so the load factor stays <= 1/2.
enum SymbBin : int {
  kSB_Zero = 0,    // row_flp == 0
  kSB_Tiny = 1,    // row_flp <= 32: one warp, one product per lane
  kSB_H1K = 2,     // t <= 512:   128 threads, 1024-slot table
  kSB_H2K = 3,     // t <= 1024:  128 threads, 2048-slot table
  kSB_H4K = 4,     // t <= 2048:  256 threads, 4096-slot table
  kSB_H8K = 5,     // t <= 4096:  256 threads, 8192-slot table (32 KiB)
  kSB_H16K = 6,    // t <= 8192:  256 threads, 16384-slot table (64 KiB)
  kSB_H32K = 7,    // t <= 16384: 512 threads, 32768-slot table (128 KiB)
  kSB_Dense = 8,   // larger: column bitmap in shared memory
  kSymbBins = 9
};

// ESC bins by products (bucketed ESC, 256 threads; capacity = the bound);
// hash bins by nnz of the row.
enum NumcBin : int {
  kNB_Zero = 0,    // no products
  kNB_Tiny = 1,    // row_flp <= 32: warp sort in registers
  kNB_E1K = 2,     // ESC, row_flp <= 1024
  kNB_E2K = 3,     // ESC, row_flp <= 2048
  kNB_E3K = 4,     // ESC, row_flp <= 3072
  kNB_E4K = 5,     // ESC, row_flp <= 4096
  kNB_E5K = 6,     // ESC, row_flp <= 4800
  kNB_E6K = 7,     // ESC, row_flp <= 6144
  kNB_E8K = 8,     // ESC, row_flp <= 8192
  kNB_H256 = 9,    // hash, nnz <= 256   (256 threads, 512 slots)
  kNB_H1K = 10,    // hash, nnz <= 1024  (256 threads, 2048 slots)
  kNB_H4K = 11,    // hash, nnz <= 4096  (512 threads, 8192 slots)
  kNB_Dense = 12,  // dense column chunks in shared memory
  kNumcBins = 13
};

enum AccumMode : int { kAccHash = 0, kAccEsc = 1, kAccHybrid = 2 };

constexpr int kDenseChunkBits = 1 << 19;   // symbolic bitmap slice: 512 Ki columns (64 KiB)
constexpr int kRankCols = 1 << 19;         // numeric dense slice: 512 Ki columns (64 + 32 + 8 KiB of bitmap and ranks)
static_assert(kRankCols == kDenseChunkBits, "the symbolic and numeric slices coincide, so bitmaps carry over");

struct Csr {
  int64_t nrow, ncol;
  const int64_t* __restrict__ rp;
  const int32_t* __restrict__ col;
  const void* __restrict__ val;
};

// Rows with fuse_lo < products <= kFusedHi run through the fused ESC kernel
// when fusion is on (fuse_lo > 0; the default lower bound is kFusedLo): no
// symbolic pass, so they sit in the symbolic zero bin.
constexpr int64_t kFusedLo = 2048;
constexpr int64_t kFusedHi = 5120;
__host__ __device__ __forceinline__ bool fused_row(int64_t flp, int fuse_lo) {
  return fuse_lo > 0 && flp > fuse_lo && flp <= kFusedHi;
}
__host__ __device__ __forceinline__ int symb_bin_of(int64_t flp, int64_t ncol, int fuse = 0) {
  if (flp <= 0 || fused_row(flp, fuse)) return kSB_Zero;
  if (flp <= 32) return kSB_Tiny;
  const int64_t t = flp < ncol ? flp : ncol;
  if (t <= 512) return kSB_H1K;
  if (t <= 1024) return kSB_H2K;
  if (t <= 2048) return kSB_H4K;
  if (t <= 4096) return kSB_H8K;
  if (t <= 8192) return kSB_H16K;
  if (t <= 16384) return kSB_H32K;
  return kSB_Dense;
}

// Accumulator choice of one row: the hybrid mode takes ESC when the row's
// compression factor flp/nnz is below the threshold, as
// ams_hybacc_numc_krnl does (src/ams/ams_utils.c:1139-1149).
// esc_max and hash_max (the tuning's limits, at most 8192 and 4096) cap the
// rows the ESC and hash kernels take; larger rows fall through to the next
// form.
__host__ __device__ __forceinline__ int numc_bin_of(int64_t flp, int64_t nz, int mode, double thres,
                                                    int esc_max = 8192, int hash_max = 4096) {
  if (flp <= 0 || nz <= 0) return kNB_Zero;
  if (flp <= 32) return kNB_Tiny;
  bool esc = mode == kAccEsc || (mode == kAccHybrid && (double)flp / (double)nz < thres);
  if (esc && flp <= esc_max) {
    if (flp <= 1024) return kNB_E1K;
    if (flp <= 2048) return kNB_E2K;
    if (flp <= 3072) return kNB_E3K;
    if (flp <= 4096) return kNB_E4K;
    if (flp <= 4800) return kNB_E5K;
    if (flp <= 6144) return kNB_E6K;
    if (flp <= 8192) return kNB_E8K;
  }
  if (nz <= hash_max) {
    if (nz <= 256) return kNB_H256;
    if (nz <= 1024) return kNB_H1K;
    if (nz <= 4096) return kNB_H4K;
  }
  return kNB_Dense;
}

}  // namespace cas
