// casgemm kernel bodies (contracts in cas_kernels.cuh).
#include "cas_kernels.cuh"
#include "cas_sortnet.cuh"

namespace cas {

// ===================================================================== INIT

// One warp per row of A: row_flp[i] = sum over A_i of |B_k|, the symbolic
// bin histogram, and the block-reduced total and maximum.  Columns outside
// [0, B.nrow) are reported and skipped.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_flp(Csr A, Csr B, int64_t c_ncol, int64_t* __restrict__ row_flp,
      unsigned long long* __restrict__ totals, unsigned long long* __restrict__ bin_count,
      DevStatus* st, int fuse, unsigned long long* __restrict__ fused_sums) {
  __shared__ unsigned long long s_cnt[kSymbBins];
  __shared__ unsigned long long s_tot, s_max, s_f[4];
  unsigned long long my_f[4] = {0, 0, 0, 0};
  if (threadIdx.x < kSymbBins) s_cnt[threadIdx.x] = 0;
  if (threadIdx.x < 4) s_f[threadIdx.x] = 0;
  if (threadIdx.x == 0) { s_tot = 0; s_max = 0; }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * BLOCK) >> 5;
  unsigned long long my_tot = 0, my_max = 0;
  for (int64_t r = ((int64_t)blockIdx.x * BLOCK + threadIdx.x) >> 5; r < A.nrow; r += nw) {
    const int64_t s = A.rp[r], e = A.rp[r + 1];
    long long sum = 0;
    for (int64_t j = s + lane; j < e; j += 32) {
      const int32_t k = A.col[j];
      if ((uint64_t)k >= (uint64_t)B.nrow) {
        dev_report(st, kDevBadIndex, 0, r);
        continue;
      }
      sum += B.rp[k + 1] - B.rp[k];
    }
    sum = warp_sum(sum);
    if (lane == 0) {
      row_flp[r] = sum;
      my_tot += (unsigned long long)sum;
      my_max = max(my_max, (unsigned long long)sum);
      atomicAdd(&s_cnt[symb_bin_of(sum, c_ncol, fuse)], 1ull);
      if (fused_row(sum, fuse)) {  // fused rows: count, products, output bound, nnz(A)
        my_f[0] += 1;
        my_f[1] += (unsigned long long)sum;
        my_f[2] += (unsigned long long)(sum < c_ncol ? sum : c_ncol);
        my_f[3] += (unsigned long long)(e - s);
      }
    }
  }
  if (lane == 0 && my_f[0])
    for (int i = 0; i < 4; ++i) atomicAdd(&s_f[i], my_f[i]);
  if (lane == 0) {
    atomicAdd(&s_tot, my_tot);
    atomicMax(&s_max, my_max);
  }
  __syncthreads();
  if (threadIdx.x < kSymbBins && s_cnt[threadIdx.x]) atomicAdd(&bin_count[threadIdx.x], s_cnt[threadIdx.x]);
  if (threadIdx.x < 4 && s_f[threadIdx.x]) atomicAdd(&fused_sums[threadIdx.x], s_f[threadIdx.x]);
  if (threadIdx.x == 0) {
    atomicAdd(&totals[0], s_tot);
    atomicMax(&totals[1], s_max);
  }
}

// The sum over A's rows of min(products, c_ncol), a bound on nnz(C) that is
// known before any row is counted (C in host memory by row blocks takes its
// host arrays by it).  A warp per row; columns outside [0, B.nrow) are
// skipped (the input check reports them).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_nnz_bound(Csr A, Csr B, int64_t c_ncol, unsigned long long* __restrict__ bound) {
  __shared__ unsigned long long s_b;
  if (threadIdx.x == 0) s_b = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * BLOCK) >> 5;
  unsigned long long my_b = 0;
  for (int64_t r = ((int64_t)blockIdx.x * BLOCK + threadIdx.x) >> 5; r < A.nrow; r += nw) {
    long long sum = 0;
    for (int64_t j = A.rp[r] + lane; j < A.rp[r + 1]; j += 32) {
      const int32_t k = A.col[j];
      if ((uint64_t)k < (uint64_t)B.nrow) sum += B.rp[k + 1] - B.rp[k];
    }
    sum = warp_sum(sum);
    my_b += (unsigned long long)(sum < c_ncol ? sum : c_ncol);
  }
  if (lane == 0 && my_b) atomicAdd(&s_b, my_b);
  __syncthreads();
  if (threadIdx.x == 0 && s_b) atomicAdd(bound, s_b);
}

// dst[0..n) = src[0..n) + add (a row block's row pointers moved to their
// place in C's).
__global__ void k_rebase_to(int64_t* __restrict__ dst, const int64_t* __restrict__ src, int64_t n, int64_t add) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i] + add;
}

// n 8-byte words from device memory into pinned host memory that the device
// maps (dst is the mapping's device-side address).  The words cross the host
// link as the kernel's stores, not as a copy-engine transfer, so they do not
// queue behind bulk copies to the host that are in flight on other streams.
__global__ void k_fetch_words(unsigned long long* __restrict__ dst, const unsigned long long* __restrict__ src,
                              int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Rows into per-bin lists.  cursor[b] starts at the bin's offset; lanes that
// hit the same bin share one atomic (warp-aggregated).
__global__ void k_bin_scatter_symb(int64_t m, const int64_t* __restrict__ row_flp, int64_t c_ncol,
                                   unsigned long long* __restrict__ cursor, int32_t* __restrict__ rows, int fuse) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int b = symb_bin_of(row_flp[r], c_ncol, fuse);
    const unsigned long long pos = warp_aggregated_add(cursor, b);
    rows[pos] = (int32_t)r;
  }
}

// Fused rows in ascending order: a 0/1 mark per row, scanned, then scattered.
__global__ void k_fused_mark(int64_t m, const int64_t* __restrict__ row_flp, int fuse, int64_t* __restrict__ mark) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x)
    mark[r] = fused_row(row_flp[r], fuse) ? 1 : 0;
}
__global__ void k_fused_scatter(int64_t m, const int64_t* __restrict__ row_flp, int fuse,
                                const int64_t* __restrict__ pos, int32_t* __restrict__ frows) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x)
    if (fused_row(row_flp[r], fuse)) frows[pos[r]] = (int32_t)r;
}

// Numeric bin histogram plus, per bin, the sums of products, nnz(C) and
// nnz(A) of its rows (for the per-kernel algorithmic byte count).
// Heavy rows launch heaviest first (longest-processing-time order, so the
// largest rows do not start last and run alone): within the dense bin, rows
// are grouped by floor(log2(products)), the largest group first.
constexpr int kHeavyClasses = 48;
__device__ __forceinline__ int heavy_class(int64_t flp) {  // 0 for the heaviest rows
  const int l = 63 - __clzll((unsigned long long)flp);
  return l >= kHeavyClasses ? 0 : kHeavyClasses - 1 - l;
}

__global__ void k_bin_count_numc(int64_t m, const int64_t* __restrict__ row_flp, const int64_t* __restrict__ crp,
                                 const int64_t* __restrict__ arp, int mode, double thres, int esc_max, int hash_max,
                                 unsigned long long* __restrict__ bin_count, unsigned long long* __restrict__ bin_sums,
                                 unsigned long long* __restrict__ heavy_count) {
  __shared__ unsigned long long s_cnt[4 * kNumcBins];
  __shared__ unsigned long long s_heavy[kHeavyClasses];
  if (threadIdx.x < 4 * kNumcBins) s_cnt[threadIdx.x] = 0;
  if (threadIdx.x < kHeavyClasses) s_heavy[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t flp = row_flp[r], nz = crp[r + 1] - crp[r];
    const int b = numc_bin_of(flp, nz, mode, thres, esc_max, hash_max);
    if (b == kNB_Dense) atomicAdd(&s_heavy[heavy_class(flp)], 1ull);
    atomicAdd(&s_cnt[b], 1ull);
    atomicAdd(&s_cnt[kNumcBins + b], (unsigned long long)flp);
    atomicAdd(&s_cnt[2 * kNumcBins + b], (unsigned long long)nz);
    atomicAdd(&s_cnt[3 * kNumcBins + b], (unsigned long long)(arp[r + 1] - arp[r]));
  }
  __syncthreads();
  if (threadIdx.x < kNumcBins && s_cnt[threadIdx.x]) atomicAdd(&bin_count[threadIdx.x], s_cnt[threadIdx.x]);
  if (threadIdx.x >= kNumcBins && threadIdx.x < 4 * kNumcBins && s_cnt[threadIdx.x])
    atomicAdd(&bin_sums[threadIdx.x - kNumcBins], s_cnt[threadIdx.x]);
  if (threadIdx.x < kHeavyClasses && s_heavy[threadIdx.x]) atomicAdd(&heavy_count[threadIdx.x], s_heavy[threadIdx.x]);
}

__global__ void k_bin_scatter_numc(int64_t m, const int64_t* __restrict__ row_flp, const int64_t* __restrict__ crp,
                                   int mode, double thres, int esc_max, int hash_max,
                                   unsigned long long* __restrict__ cursor,
                                   unsigned long long* __restrict__ heavy_cursor, int32_t* __restrict__ rows) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t flp = row_flp[r];
    const int b = numc_bin_of(flp, crp[r + 1] - crp[r], mode, thres, esc_max, hash_max);
    const unsigned long long pos =
        b == kNB_Dense ? warp_aggregated_add(heavy_cursor, heavy_class(flp)) : warp_aggregated_add(cursor, b);
    rows[pos] = (int32_t)r;
  }
}

// ===================================================================== scan
// Exclusive scan out[0..n) of in[0..n-1): out[0] = 0, out[i+1] = out[i] + in[i]
// (the contract of scan, src/mm/mm_utils.c:903-911).  Reduce-then-scan over
// tiles of BLOCK*ITEMS: no inter-block waiting.
constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__global__ void __launch_bounds__(kScanBlock)
k_scan_partials(const int64_t* __restrict__ in, int64_t n_in, int64_t* __restrict__ partial) {
  __shared__ long long tmp[kScanBlock / 32 + 1];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  long long s = 0;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    const int64_t i = base + (int64_t)u * kScanBlock + threadIdx.x;
    if (i < n_in) s += in[i];
  }
  s = block_sum<kScanBlock, long long>(s, tmp);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// single block: exclusive scan of the tile partials (any count, in rounds)
__global__ void __launch_bounds__(kScanBlock)
k_scan_top(int64_t* __restrict__ partial, int64_t nparts, int64_t* __restrict__ total_out) {
  __shared__ long long tmp[kScanBlock / 32 + 1];
  long long carry = 0;
  for (int64_t b0 = 0; b0 < nparts; b0 += kScanBlock) {
    const int64_t i = b0 + threadIdx.x;
    const long long v = i < nparts ? partial[i] : 0;
    long long tot;
    const long long ex = block_exclusive_sum<kScanBlock, long long>(v, tmp, tot);
    if (i < nparts) partial[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void __launch_bounds__(kScanBlock)
k_scan_apply(const int64_t* __restrict__ in, int64_t n_in, const int64_t* __restrict__ partial,
             int64_t* __restrict__ out, int64_t n_out) {
  __shared__ long long tmp[kScanBlock / 32 + 1];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  long long v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    const int64_t i = base + u;
    v[u] = i < n_in ? in[i] : 0;
    s += v[u];
  }
  long long tot;
  long long run = block_exclusive_sum<kScanBlock, long long>(s, tmp, tot) + partial[blockIdx.x];
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    const int64_t i = base + u;
    if (i < n_out) out[i] = run;
    run += v[u];
  }
}

// ============================================================ row expansion
// Enumerates the products of one row of A*B inside a thread block: A entries
// are staged min(BLOCK, kAChunk) at a time (B row start, length, A value), their lengths
// scanned, and each thread then takes products p = tid, tid+BLOCK, ... and
// finds its A entry by binary search, so work is balanced whatever the B row
// lengths.  Loads of U products are issued before any is consumed.  With
// `ranged`, every B row is cut to the columns [c0, c1) by binary search (B
// rows sorted); otherwise f receives every product.
constexpr int kAChunk = 256;
constexpr int kUnroll = 8;

template <typename VIn>
struct alignas(16) Stage {
  int64_t bs[kAChunk];
  int64_t pre[kAChunk + 1];
  VIn av[kAChunk];
  long long tmp[33];
};

template <int BLOCK, bool NEED_VAL, typename VIn, typename F>
__device__ __forceinline__ int64_t expand_entries(const Csr& A, const Csr& B, int64_t as, int64_t ae, Stage<VIn>& sg,
                                                  bool ranged, int32_t c0, int32_t c1, F&& f) {
  const VIn* __restrict__ aval = static_cast<const VIn*>(A.val);
  const VIn* __restrict__ bval = static_cast<const VIn*>(B.val);
  constexpr int ACH = BLOCK < kAChunk ? BLOCK : kAChunk;  // one staged A entry per thread
  int64_t pbase = 0;
  for (int64_t a0 = as; a0 < ae; a0 += ACH) {
    const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
    long long len = 0;
    if (threadIdx.x < na) {
      const int32_t k = A.col[a0 + threadIdx.x];
      int64_t lo = B.rp[k], hi = B.rp[k + 1];
      if (ranged) {
        lo = lower_bound_g(B.col, lo, hi, c0);
        hi = lower_bound_g(B.col, lo, hi, c1);
      }
      sg.bs[threadIdx.x] = lo;
      len = hi - lo;
      if (NEED_VAL) sg.av[threadIdx.x] = aval[a0 + threadIdx.x];
    }
    long long total;
    const long long ex = block_exclusive_sum<BLOCK, long long>(len, sg.tmp, total);
    if (threadIdx.x < ACH) sg.pre[threadIdx.x] = ex;
    if (threadIdx.x == 0) sg.pre[na] = total;
    __syncthreads();
    // A entry of product p: the interpolated guess p * na / total, checked
    // with its neighbours (exact for rows of near-equal B row lengths), else
    // a binary search for the last entry whose prefix is <= p.
    const float per = total > 0 ? (float)na / (float)total : 0.f;
    for (int64_t p0 = threadIdx.x; p0 < total; p0 += (int64_t)BLOCK * kUnroll) {
      int32_t key[kUnroll];
      VIn bv[kUnroll];
      int sgi[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int64_t p = p0 + (int64_t)u * BLOCK;
        sgi[u] = -1;
        if (p < total) {
          int s = min(na - 1, (int)((float)p * per));
          if (sg.pre[s] > p) {
            if (s > 0 && sg.pre[s - 1] <= p) {
              --s;
            } else {
              int lo = 0, hi = s;
              while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (sg.pre[mid] <= p) lo = mid; else hi = mid;
              }
              s = lo;
            }
          } else if (sg.pre[s + 1] <= p) {
            if (sg.pre[s + 2] > p) {
              ++s;
            } else {
              int lo = s + 2, hi = na;
              while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (sg.pre[mid] <= p) lo = mid; else hi = mid;
              }
              s = lo;
            }
          }
          const int lo = s;
          const int64_t j = sg.bs[lo] + (p - sg.pre[lo]);
          key[u] = __ldg(B.col + j);
          if (NEED_VAL) bv[u] = __ldg(bval + j);
          sgi[u] = lo;
        }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (sgi[u] >= 0) {
          if (!ranged || (key[u] >= c0 && key[u] < c1)) {
            if (NEED_VAL) f(key[u], sg.av[sgi[u]], bv[u], pbase + p0 + (int64_t)u * BLOCK);
            else f(key[u], VIn(0), VIn(0), pbase + p0 + (int64_t)u * BLOCK);
          }
        }
      }
    }
    pbase += total;
    __syncthreads();
  }
  return pbase;
}

// The products of row r (its A entries [A.rp[r], A.rp[r + 1])).
template <int BLOCK, bool NEED_VAL, typename VIn, typename F>
__device__ __forceinline__ int64_t expand_row(const Csr& A, const Csr& B, int64_t r, Stage<VIn>& sg,
                                              bool ranged, int32_t c0, int32_t c1, F&& f) {
  return expand_entries<BLOCK, NEED_VAL, VIn>(A, B, A.rp[r], A.rp[r + 1], sg, ranged, c0, c1, f);
}

// ================================================================ SYMBOLIC

// Rows with at most 32 products: one warp per row, one product per lane; the
// distinct count is the number of lanes that lead their __match_any_sync group.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_symb_tiny(const int32_t* __restrict__ rows, int64_t nrows, Csr A, Csr B, int64_t* __restrict__ row_nz,
            DevStatus* st) {
  __shared__ int64_t s_bs[BLOCK];
  __shared__ int32_t s_ex[BLOCK];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int64_t* wbs = s_bs + wib * 32;
  int32_t* wex = s_ex + wib * 32;
  const int64_t w = ((int64_t)blockIdx.x * BLOCK + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int64_t r = rows[w];
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  uint64_t mykey = (1ull << 32) | (uint64_t)lane;  // unique dummy for empty lanes
  int base = 0;
  for (int64_t a0 = as; a0 < ae; a0 += 32) {
    const int64_t ja = a0 + lane;
    int32_t len = 0;
    int64_t bs = 0;
    if (ja < ae) {
      const int32_t k = A.col[ja];
      bs = B.rp[k];
      len = (int32_t)(B.rp[k + 1] - bs);
    }
    const int32_t inc = warp_inclusive_sum(len);
    const int32_t tot = __shfl_sync(kFull, inc, 31);
    wbs[lane] = bs;
    wex[lane] = inc - len;
    __syncwarp();
    const int p = lane - base;
    if (p >= 0 && p < tot) {
      int lo = 0, hi = 32;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (wex[mid] <= p) lo = mid; else hi = mid;
      }
      mykey = (uint64_t)(uint32_t)__ldg(B.col + wbs[lo] + (p - wex[lo]));
    }
    base += tot;
    __syncwarp();
  }
  if (base > 32 && lane == 0) dev_report(st, kDevCapacity, 1, r);
  const unsigned peers = __match_any_sync(kFull, mykey);
  const bool lead = (mykey >> 32) == 0 && lane == __ffs(peers) - 1;
  const int cnt = __popc(__ballot_sync(kFull, lead));
  if (lane == 0) row_nz[r] = cnt;
}

// Column range [lo, hi) that row r of A*B can reach: with B's rows sorted,
// from the first and last column of every B row the row gathers; otherwise
// [0, ncol).  Block-wide; every thread gets the range.
template <int BLOCK>
__device__ __forceinline__ void row_col_range(const Csr& A, const Csr& B, int64_t r, bool b_sorted, int64_t ncol,
                                              int64_t& lo, int64_t& hi) {
  __shared__ uint32_t red[2];
  if (!b_sorted) {
    lo = 0;
    hi = ncol;
    return;
  }
  if (threadIdx.x == 0) { red[0] = 0xFFFFFFFFu; red[1] = 0u; }
  __syncthreads();
  uint32_t mn = 0xFFFFFFFFu, mx = 0u;
  const int64_t ae = A.rp[r + 1];
  for (int64_t j = A.rp[r] + threadIdx.x; j < ae; j += BLOCK) {
    const int32_t k = A.col[j];
    const int64_t s = B.rp[k], e = B.rp[k + 1];
    if (e > s) {
      mn = min(mn, (uint32_t)__ldg(B.col + s));
      mx = max(mx, (uint32_t)__ldg(B.col + e - 1));
    }
  }
  mn = warp_min_u32(mn);
  mx = warp_max_u32(mx);
  if ((threadIdx.x & 31) == 0 && mx >= mn) {
    atomicMin(&red[0], mn);
    atomicMax(&red[1], mx);
  }
  __syncthreads();
  if (red[1] >= red[0]) {
    lo = red[0];
    hi = (int64_t)red[1] + 1;
  } else {
    lo = hi = 0;
  }
  __syncthreads();
}

// Heavy rows: a bitmap over kDenseChunkBits columns at a time, one pass per
// chunk of the row's column range; the count is the population count.  B
// rows are cut to each column chunk by binary search when there is more than
// one chunk.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_symb_dense(const int32_t* __restrict__ rows, Csr A, Csr B, int64_t c_ncol, int32_t b_sorted,
             int64_t* __restrict__ row_nz, uint32_t* __restrict__ saved, int32_t* __restrict__ saved_slot,
             int saved_slices, DevStatus* st) {
  constexpr int W = kDenseChunkBits / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem);
  Stage<double>& sg = *reinterpret_cast<Stage<double>*>(smem + W * sizeof(uint32_t));
  const int64_t r = rows[blockIdx.x];
  int64_t lo, hi;
  row_col_range<BLOCK>(A, B, r, b_sorted != 0, c_ncol, lo, hi);
  const bool multi = hi - lo > kDenseChunkBits;
  long long cnt = 0;
  for (int64_t c0 = lo; c0 < hi; c0 += kDenseChunkBits) {
    const int64_t c1 = (hi < c0 + kDenseChunkBits ? hi : c0 + kDenseChunkBits);
    const int nw = (int)((c1 - c0 + 31) >> 5);  // words the slice uses
    for (int i = threadIdx.x; i < nw; i += BLOCK) bm[i] = 0u;
    __syncthreads();
    bool bad = false;
    expand_row<BLOCK, false, double>(A, B, r, sg, multi, (int32_t)c0, (int32_t)c1,
                                     [&](int32_t key, double, double, int64_t) {
      const int64_t idx = (int64_t)key - c0;
      if (idx < 0 || idx >= kDenseChunkBits) { bad = true; return; }
      atomicOr(&bm[idx >> 5], 1u << (idx & 31));
    });
    if (bad && !multi) dev_report(st, kDevBadIndex, 3, r);
    __syncthreads();
    for (int i = threadIdx.x; i < nw; i += BLOCK) cnt += __popc(bm[i]);
    // keep the bitmap for the numeric kernel when the row's slices fit its
    // saved_slices slots (the symbolic and numeric slices are the same: both
    // kDenseChunkBits == kRankCols columns from the row's first column)
    const int nsl = (int)((hi - lo + kRankCols - 1) / kRankCols);
    if (saved && nsl <= saved_slices) {
      const int sl = (int)((c0 - lo) / kRankCols);
      uint32_t* dst = saved + ((size_t)blockIdx.x * saved_slices + sl) * (kRankCols / 32);
      for (int i = threadIdx.x; i < nw; i += BLOCK) dst[i] = bm[i];
      if (threadIdx.x == 0) saved_slot[r] = (int32_t)blockIdx.x;
    }
    __syncthreads();
  }
  cnt = block_sum<BLOCK, long long>(cnt, sg.tmp);
  if (threadIdx.x == 0) row_nz[r] = cnt;
}

// ================================================================= NUMERIC

// Rows with at most 32 products: one product per lane, a 32-lane bitonic sort
// by column in registers, a segmented sum from the right, and one store per
// distinct column (the ESC accumulator at warp scale).
template <int BLOCK, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_numc_tiny(const int32_t* __restrict__ rows, int64_t nrows, Csr A, Csr B, const int64_t* __restrict__ crp,
            int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval, DevStatus* st) {
  using AT = typename Acc<VIn>::T;
  __shared__ int64_t s_bs[BLOCK];
  __shared__ int32_t s_ex[BLOCK];
  __shared__ VIn s_av[BLOCK];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int64_t* wbs = s_bs + wib * 32;
  int32_t* wex = s_ex + wib * 32;
  VIn* wav = s_av + wib * 32;
  const int64_t w = ((int64_t)blockIdx.x * BLOCK + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int64_t r = rows[w];
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  const VIn* __restrict__ aval = static_cast<const VIn*>(A.val);
  const VIn* __restrict__ bval = static_cast<const VIn*>(B.val);
  uint32_t key = kEmptyKey;
  AT val = AT(0);
  int base = 0;
  for (int64_t a0 = as; a0 < ae; a0 += 32) {
    const int64_t ja = a0 + lane;
    int32_t len = 0;
    int64_t bs = 0;
    VIn av = VIn(0);
    if (ja < ae) {
      const int32_t k = A.col[ja];
      bs = B.rp[k];
      len = (int32_t)(B.rp[k + 1] - bs);
      av = aval[ja];
    }
    const int32_t inc = warp_inclusive_sum(len);
    const int32_t tot = __shfl_sync(kFull, inc, 31);
    wbs[lane] = bs;
    wex[lane] = inc - len;
    wav[lane] = av;
    __syncwarp();
    const int p = lane - base;
    if (p >= 0 && p < tot) {
      int lo = 0, hi = 32;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (wex[mid] <= p) lo = mid; else hi = mid;
      }
      const int64_t j = wbs[lo] + (p - wex[lo]);
      key = (uint32_t)__ldg(B.col + j);
      val = Acc<VIn>::mul(wav[lo], __ldg(bval + j));
    }
    base += tot;
    __syncwarp();
  }
  // bitonic sort of (key, val) across the warp, ascending by key
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const uint32_t ok = __shfl_xor_sync(kFull, key, j);
      const AT ov = __shfl_xor_sync(kFull, val, j);
      const bool up = (lane & k) == 0;
      const bool lower = (lane & j) == 0;
      const bool take = lower ? (up ? ok < key : ok > key) : (up ? ok > key : ok < key);
      if (take) { key = ok; val = ov; }
    }
  }
  // segmented sum toward each run's first lane
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t ok = __shfl_down_sync(kFull, key, d);
    const AT ov = __shfl_down_sync(kFull, val, d);
    if (lane + d < 32 && ok == key) val += ov;
  }
  const uint32_t prev = __shfl_up_sync(kFull, key, 1);
  const bool head = key != kEmptyKey && (lane == 0 || prev != key);
  const unsigned heads = __ballot_sync(kFull, head);
  const int64_t c0 = crp[r], nz = crp[r + 1] - c0;
  const int pos = __popc(heads & lanemask_lt());
  if (head && pos < nz) {
    ccol[c0 + pos] = (int32_t)key;
    cval[c0 + pos] = val;
  }
  if (lane == 0 && __popc(heads) != nz) dev_report(st, __popc(heads) > nz ? kDevRowOverflow : kDevRowUnderflow, 10, r);
}

// Shared-memory layout helpers for the sort-based kernels.
template <int BLOCK>
struct alignas(16) SortScratch {
  uint16_t hist[(BLOCK / 32) * 256];
  int tmp[33];
};

// ESC accumulator for rows of at most CAP products: expand (column, a*b) into
// shared memory, sort by column with the block radix sort, and sum runs of
// equal columns (ams_hsersc_numc_krnl, src/ams/ams_utils.c:399-456).  The
// sort is stable, so each sum is taken in expansion order.
template <int BLOCK, int CAP, typename VIn>
__device__ __forceinline__ void esc_radix_row(int64_t r, const Csr& A, const Csr& B, const int64_t* __restrict__ crp,
                                              int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval,
                                              DevStatus* st, uint8_t* smem) {
  using AT = typename Acc<VIn>::T;
  uint64_t* items = reinterpret_cast<uint64_t*>(smem);
  uint64_t* items2 = items + CAP;
  AT* ev = reinterpret_cast<AT*>(items2 + CAP);
  SortScratch<BLOCK>& ss = *reinterpret_cast<SortScratch<BLOCK>*>(ev + CAP);
  Stage<VIn>& sg = *reinterpret_cast<Stage<VIn>*>(reinterpret_cast<uint8_t*>(&ss) + sizeof(SortScratch<BLOCK>));
  __shared__ uint32_t s_min, s_max;
  __shared__ int s_over;
  if (threadIdx.x == 0) { s_min = 0xFFFFFFFFu; s_max = 0u; s_over = 0; }
  __syncthreads();
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u;
  bool over = false;
  const int64_t n = expand_row<BLOCK, true, VIn>(A, B, r, sg, false, 0, 0,
                                                [&](int32_t key, VIn av, VIn bv, int64_t p) {
    if (p >= CAP) { over = true; return; }
    items[p] = ((uint64_t)(uint32_t)key << 32) | (uint64_t)p;
    ev[p] = Acc<VIn>::mul(av, bv);
    kmin = min(kmin, (uint32_t)key);
    kmax = max(kmax, (uint32_t)key);
  });
  kmin = warp_min_u32(kmin);
  kmax = warp_max_u32(kmax);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&s_min, kmin);
    atomicMax(&s_max, kmax);
    if (over) s_over = 1;
  }
  __syncthreads();
  const int64_t c0 = crp[r], nz = crp[r + 1] - c0;
  if (s_over || n > CAP) {
    if (threadIdx.x == 0) dev_report(st, kDevCapacity, 11, r);
    return;
  }
  const int nn = (int)n;
  const uint64_t* sorted = block_radix_sort<BLOCK>(items, items2, nn, s_min, s_max, ss.hist, ss.tmp);
  int carry = 0;
  for (int t0 = 0; t0 < nn; t0 += BLOCK) {
    const int t = t0 + threadIdx.x;
    uint32_t key = 0;
    bool head = false;
    if (t < nn) {
      key = (uint32_t)(sorted[t] >> 32);
      head = t == 0 || (uint32_t)(sorted[t - 1] >> 32) != key;
    }
    int tot;
    const int ex = block_exclusive_sum<BLOCK, int>(head ? 1 : 0, ss.tmp, tot);
    if (head) {
      AT sum = ev[(uint32_t)sorted[t]];
      for (int t2 = t + 1; t2 < nn && (uint32_t)(sorted[t2] >> 32) == key; ++t2) sum += ev[(uint32_t)sorted[t2]];
      const int64_t pos = carry + ex;
      if (pos < nz) {
        ccol[c0 + pos] = (int32_t)key;
        cval[c0 + pos] = sum;
      }
    }
    carry += tot;
  }
  if (threadIdx.x == 0 && carry != nz) dev_report(st, carry > nz ? kDevRowOverflow : kDevRowUnderflow, 11, r);
}

template <int BLOCK, int CAP, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_numc_esc(const int32_t* __restrict__ rows, Csr A, Csr B, const int64_t* __restrict__ crp,
           int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval, DevStatus* st) {
  extern __shared__ __align__(16) uint8_t smem[];
  esc_radix_row<BLOCK, CAP, VIn>(rows[blockIdx.x], A, B, crp, ccol, cval, st, smem);
}

// Persistent form for the rows the bucketed ESC kernel hands back (their
// keys fall unevenly into its buckets): the list length is read on the device.
template <int BLOCK, int CAP, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_numc_esc_overflow(const int32_t* __restrict__ rows, const unsigned int* __restrict__ count, Csr A, Csr B,
                    const int64_t* __restrict__ crp, int32_t* __restrict__ ccol,
                    typename Acc<VIn>::T* __restrict__ cval, DevStatus* st) {
  extern __shared__ __align__(16) uint8_t smem[];
  const unsigned n = *count;
  for (unsigned i = blockIdx.x; i < n; i += gridDim.x) {
    esc_radix_row<BLOCK, CAP, VIn>(rows[i], A, B, crp, ccol, cval, st, smem);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Row expansion for the capacity-bounded kernels (a row's products fit in
// shared memory).  A entries are staged kBChunk at a time; each chunk's
// product-to-entry map is a byte table written once per B row with coalesced
// stores, so finding a product's A entry is one shared-memory byte load, and
// all product indices are 32-bit.  When B's rows are sorted, the row's column
// range [kmin, kmax] is known from each B row's first and last column before
// any product is read.
constexpr int kBChunk = 128;  // A entries per staged chunk (uniform R-MAT rows have ~64)

template <typename VIn>
struct alignas(16) StageB {
  int64_t bs[kBChunk];       // start of the B row (global index)
  int32_t pre[kBChunk + 1];  // exclusive prefix of B row lengths in the chunk
  VIn av[kBChunk];
  int tmp[34];
  uint32_t kmin, kmax;
  int over;
};

// Stages one chunk of A entries [a0, a0+na) and fills segof; returns the
// chunk's product count.  With `range`, also reduces the first/last columns
// of the B rows into sg.kmin / sg.kmax (B rows sorted by column).
template <int BLOCK, bool NEED_VAL, typename VIn>
__device__ __forceinline__ int stage_chunk(const Csr& A, const Csr& B, int64_t a0, int na, StageB<VIn>& sg,
                                           uint8_t* __restrict__ segof, int cap, bool range) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  int len = 0;
  uint32_t lo_key = 0xFFFFFFFFu, hi_key = 0u;
  if (threadIdx.x < na) {
    const int32_t k = A.col[a0 + threadIdx.x];
    const int64_t lo = B.rp[k], hi = B.rp[k + 1];
    sg.bs[threadIdx.x] = lo;
    len = (int)(hi - lo);
    if (NEED_VAL) sg.av[threadIdx.x] = static_cast<const VIn*>(A.val)[a0 + threadIdx.x];
    if (range && hi > lo) {
      lo_key = (uint32_t)__ldg(B.col + lo);
      hi_key = (uint32_t)__ldg(B.col + hi - 1);
    }
  }
  if (range) {
    lo_key = warp_min_u32(lo_key);
    hi_key = warp_max_u32(hi_key);
    if (lane == 0 && hi_key >= lo_key) {
      atomicMin(&sg.kmin, lo_key);
      atomicMax(&sg.kmax, hi_key);
    }
  }
  int total;
  const int ex = block_exclusive_sum<BLOCK, int>(len, sg.tmp, total);
  if (threadIdx.x < na) sg.pre[threadIdx.x] = ex;
  if (threadIdx.x == 0) sg.pre[na] = total;
  __syncthreads();
  if (total <= cap) {
    for (int sgi = warp; sgi < na; sgi += NW) {
      const int b0 = sg.pre[sgi], l = sg.pre[sgi + 1] - b0;
      for (int i = lane; i < l; i += 32) segof[b0 + i] = (uint8_t)sgi;
    }
  }
  __syncthreads();
  return total;
}

// Product p (< total) of the staged chunk: calls f(key, a, b, p).  Loads of
// kUnroll products are issued before any is consumed.
template <int BLOCK, bool NEED_VAL, typename VIn, typename F>
__device__ __forceinline__ void expand_chunk(const Csr& B, int total, const StageB<VIn>& sg,
                                             const uint8_t* __restrict__ segof, F&& f) {
  const VIn* __restrict__ bval = static_cast<const VIn*>(B.val);
  for (int p0 = threadIdx.x; p0 < total; p0 += BLOCK * kUnroll) {
    int32_t key[kUnroll];
    VIn bv[kUnroll];
    int sgi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int p = p0 + u * BLOCK;
      sgi[u] = -1;
      if (p < total) {
        const int s = segof[p];
        const int64_t j = sg.bs[s] + (p - sg.pre[s]);
        key[u] = __ldg(B.col + j);
        if (NEED_VAL) bv[u] = __ldg(bval + j);
        sgi[u] = s;
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (sgi[u] >= 0) f(key[u], NEED_VAL ? sg.av[sgi[u]] : VIn(0), NEED_VAL ? bv[u] : VIn(0), p0 + u * BLOCK);
    }
  }
}

// Two 16-bit bucket counters per 32-bit word (shared-memory atomics are
// 32-bit); counts and offsets stay below 2^16 because CAP <= 32768.
__device__ __forceinline__ uint32_t bucket_add(uint32_t* w, int b) {
  const uint32_t sh = (b & 1) << 4;
  return (atomicAdd(&w[b >> 1], 1u << sh) >> sh) & 0xFFFFu;
}
__device__ __forceinline__ uint32_t bucket_get(const uint32_t* w, int b) { return (w[b >> 1] >> ((b & 1) << 4)) & 0xFFFFu; }

// Products of a staged chunk too large for the byte table: the A entry of
// product p is found by binary search over the 32-bit prefixes.
template <int BLOCK, typename VIn, typename F>
__device__ __forceinline__ void expand_chunk_search(const Csr& B, int na, int total, const StageB<VIn>& sg, F&& f) {
  for (int p0 = threadIdx.x; p0 < total; p0 += BLOCK * kUnroll) {
    int32_t key[kUnroll];
    bool ok[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int p = p0 + u * BLOCK;
      ok[u] = p < total;
      if (ok[u]) {
        int lo = 0, hi = na;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (sg.pre[mid] <= p) lo = mid; else hi = mid;
        }
        key[u] = __ldg(B.col + sg.bs[lo] + (p - sg.pre[lo]));
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (ok[u]) f(key[u]);
  }
}

// Symbolic phase for rows whose distinct columns fit a shared-memory hash of
// 2^TBITS keys (at least twice the bound min(row_flp, num_col)): linear
// probing on 32-bit keys, claiming a slot with atomicCAS directly (most
// products bring a new column in the rows this serves); the count is the
// number of successful claims (ams_hash_symb_krnl, src/ams/ams_utils.c:101-164,
// in shared memory).  A chunk of at most SEGCAP products uses the byte table
// to map products to A entries, a larger one binary search.
template <int BLOCK, int TBITS, int SEGCAP>
__global__ void __launch_bounds__(BLOCK)
k_symb_hash(const int32_t* __restrict__ rows, Csr A, Csr B, int64_t* __restrict__ row_nz, DevStatus* st) {
  constexpr int T = 1 << TBITS;
  constexpr int ACH = BLOCK < kBChunk ? BLOCK : kBChunk;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* tab = reinterpret_cast<uint32_t*>(smem);
  uint8_t* segof = reinterpret_cast<uint8_t*>(tab + T);
  StageB<double>& sg = *reinterpret_cast<StageB<double>*>(segof + SEGCAP);
  const int64_t r = rows[blockIdx.x];
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  for (int i = threadIdx.x; i < T / 4; i += BLOCK) reinterpret_cast<uint4*>(tab)[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
  __syncthreads();
  int cnt = 0;
  bool full = false;
  auto insert = [&](int32_t key) {
    uint32_t h = hash_slot((uint32_t)key, TBITS);
    for (int probe = 0; probe < T; ++probe) {
      const uint32_t old = atomicCAS(&tab[h], kEmptyKey, (uint32_t)key);
      if (old == kEmptyKey) { ++cnt; return; }
      if (old == (uint32_t)key) return;
      h = (h + 1) & (T - 1);
    }
    full = true;
  };
  for (int64_t a0 = as; a0 < ae; a0 += ACH) {
    const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
    const int total = stage_chunk<BLOCK, false, double>(A, B, a0, na, sg, segof, SEGCAP, false);
    if (total <= SEGCAP)
      expand_chunk<BLOCK, false, double>(B, total, sg, segof, [&](int32_t key, double, double, int) { insert(key); });
    else
      expand_chunk_search<BLOCK, double>(B, na, total, sg, insert);
    __syncthreads();
  }
  if (full) dev_report(st, kDevTableFull, 2, r);
  int tot;
  block_exclusive_sum<BLOCK, int>(cnt, sg.tmp, tot);
  if (threadIdx.x == 0) row_nz[r] = tot;
}

__device__ __forceinline__ void atomic_add_sh(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_sh(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// Sorts the (key, value) pairs of one bucket [s, e), 1 <= e - s <= N, in
// shared memory by key with the N-input network of cas_sortnet.cuh on packed
// (key - kbase, slot) words, sums equal keys, and leaves the distinct (key,
// sum) pairs at [s, s + heads) and kEmptyKey behind them; returns heads.  All
// keys of the bucket lie in [kbase, kbase + 2^23).  One lane per bucket; the
// caller picks N from the largest bucket of the warp.
template <int N, typename AT>
__device__ __forceinline__ int sort_compact_small(uint32_t* __restrict__ skey, AT* __restrict__ sval, int s, int e,
                                                  uint32_t kbase) {
  const int nb = e - s;
  uint32_t w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) w[i] = i < nb ? sortnet_pack(skey[s + i] - kbase, i) : 0xFFFFFFFFu;
  sort_net(w);
  AT v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = i < nb ? sval[s + sortnet_slot(w[i])] : AT(0);
  int h = 0;
  uint32_t prev = sortnet_offset(w[0]);
  AT acc = v[0];
#pragma unroll
  for (int i = 1; i < N; ++i) {
    if (i < nb) {
      const uint32_t k = sortnet_offset(w[i]);
      if (k != prev) {
        skey[s + h] = kbase + prev;
        sval[s + h] = acc;
        ++h;
        prev = k;
        acc = v[i];
      } else {
        acc += v[i];
      }
    }
  }
  skey[s + h] = kbase + prev;
  sval[s + h] = acc;
  ++h;
  for (int i = h; i < nb; ++i) skey[s + i] = kEmptyKey;
  return h;
}

// Sorts the pairs of one bucket [s, e), e - s <= 128, by key with the whole
// warp and leaves the distinct (key, sum) pairs at [s, s + heads), kEmptyKey
// behind them; returns heads.  A rank sort (a pair's rank counts the smaller
// keys and the equal keys before it, so equal keys keep their order) puts the
// pairs in order; a segmented inclusive scan over each 32-pair row of the
// sorted order (Hillis-Steele, segments start at the first pair of each key),
// carried from row to row, gives every run's sum at its last pair.  No two
// lanes add into the same slot, so a run of one key (the diagonal column of
// A*A^T brings one per A entry) costs no more than distinct keys.
template <typename AT>
__device__ __forceinline__ int warp_sort_compact(uint32_t* __restrict__ skey, AT* __restrict__ sval, int s, int e) {
  constexpr int PER = 4;
  const int lane = threadIdx.x & 31;
  const int b = e - s;
  uint32_t k[PER];
  AT v[PER];
  int rk[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int idx = lane + 32 * i;
    k[i] = idx < b ? skey[s + idx] : kEmptyKey;
    v[i] = idx < b ? sval[s + idx] : AT(0);
    rk[i] = 0;
  }
#pragma unroll 4
  for (int j = 0; j < b; ++j) {
    const uint32_t kj = skey[s + j];
#pragma unroll
    for (int i = 0; i < PER; ++i) rk[i] += (kj < k[i]) || (kj == k[i] && j < lane + 32 * i);
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    if (lane + 32 * i < b) {
      skey[s + rk[i]] = k[i];
      sval[s + rk[i]] = v[i];
    }
  }
  __syncwarp();
  int heads = 0;
  int run[PER];
  bool hd[PER], last[PER];
  AT carry = AT(0);
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int t = lane + 32 * i;
    const bool in = t < b;
    k[i] = in ? skey[s + t] : kEmptyKey;
    AT x = in ? sval[s + t] : AT(0);
    const uint32_t kp = (t > 0 && in) ? skey[s + t - 1] : ~k[i];
    const uint32_t kn = (t + 1 < b) ? skey[s + t + 1] : ~k[i];
    hd[i] = in && k[i] != kp;
    last[i] = in && k[i] != kn;
    const unsigned m = __ballot_sync(kFull, hd[i]);
    run[i] = heads + __popc(m & ((lanemask_lt() << 1) | 1u)) - 1;
    heads += __popc(m);
    // segmented scan of the row; pairs past the bucket start segments of their own
    bool f = hd[i] || !in;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const AT y = __shfl_up_sync(kFull, x, d);
      const bool g = __shfl_up_sync(kFull, (int)f, d) != 0;
      if (lane >= d) {
        if (!f) x = y + x;
        f = f || g;
      }
    }
    if (!f) x = carry + x;  // the run continues from the previous row
    carry = __shfl_sync(kFull, x, 31);
    v[i] = x;
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    if (hd[i]) skey[s + run[i]] = k[i];
    if (last[i]) sval[s + run[i]] = v[i];
  }
  for (int t = heads + lane; t < b; t += 32) skey[s + t] = kEmptyKey;
  __syncwarp();
  return heads;
}

// ESC accumulator with a one-pass bucket sort, for rows of at most CAP
// products (ams_hsersc_numc_krnl, src/ams/ams_utils.c:399-456):
//  1. a keys-only expansion histograms the products into NB = 2^NBB buckets
//     (about four products per bucket) by the high bits of (column - min
//     column);
//  2. a second expansion writes every (column, a*b) straight to its bucket's
//     next slot, so the pairs land in bucket order with no index array;
//  3. one lane per bucket sorts the bucket by column, sums equal columns and
//     compacts them to the bucket's front (kEmptyKey behind); buckets of more
//     than 8 pairs are sorted by a whole warp each;
//  4. 32 slots at a time, warps count and then write the distinct pairs, so a
//     warp's global stores are contiguous.
// A row with a bucket of more than kBucketLimit products (columns crowded
// into a narrow range) is appended to `ovf` and left to the radix-sort ESC
// kernel.  The limit counts products, not distinct columns: the diagonal
// column of A*A^T alone puts |A_i| products into one bucket.  Shared memory:
// 13 bytes per product plus half a byte per bucket.
constexpr int kBucketLimit = 128;
// Buckets of more than kBucketLimit pairs that span at most kHugeWidth
// columns (hub columns of a skewed graph, repeated many times) are summed
// by the whole block into a dense kHugeWidth-slot array over the byte
// table, which comes out sorted; a row may have kHugeBuckets of them.
constexpr int kHugeWidth = 256;
constexpr int kHugeBuckets = 16;

// ---- fused rows: count and place in one pass -------------------------------
// The fused form of the kernel runs the rows of one product-count range
// without a symbolic pass.  Each block takes the next row in row order from
// a ticket counter, counts the row's distinct columns, and finds where the
// row goes in C from the counts of the earlier fused rows by a decoupled
// look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan with
// Decoupled Look-back", 2016) over one status word per fused row, plus the
// known counts of all other rows before it.  A block waits only for rows
// with an earlier ticket, whose blocks are already running, so the chain
// always advances; every wait is bounded all the same and gives up with an
// error status instead of hanging.
struct Fused {
  const int32_t* rows;              // fused rows, ascending
  unsigned long long* ticket;       // next ticket
  unsigned long long* status;       // one look-back word per fused row, zeroed
  const int64_t* known;             // exclusive prefix of the counts of the other rows
  int64_t* row_nz;                  // out: each fused row's count
  int64_t cap;                      // entries C has room for
};
constexpr unsigned long long kLbAgg = 1ull << 62;   // the word holds the row's own count
constexpr unsigned long long kLbInc = 2ull << 62;   // the word holds the inclusive prefix
constexpr unsigned long long kLbVal = (1ull << 62) - 1;
constexpr int kLbSpins = 1 << 22;                   // polls (about 64 ns apart) before giving up

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Warp 0 of the block holding ticket t: publishes `count`, returns the sum of
// the counts of all earlier tickets, or -1 when a wait gave up.
__device__ long long lookback_prefix(unsigned long long* status, int64_t t, long long count) {
  const int lane = threadIdx.x & 31;
  if (t == 0) {
    if (lane == 0) st_release_u64(&status[0], kLbInc | (unsigned long long)count);
    return 0;
  }
  if (lane == 0) st_release_u64(&status[t], kLbAgg | (unsigned long long)count);
  long long excl = 0;
  int64_t j = t - 1;
  int spins = 0;
  for (;;) {
    const int64_t idx = j - lane;
    const unsigned long long v = idx >= 0 ? ld_acquire_u64(&status[idx]) : kLbInc;
    if (__any_sync(kFull, (v >> 62) == 0)) {
      if (++spins > kLbSpins) return -1;
      __nanosleep(64);
      continue;
    }
    const unsigned inc = __ballot_sync(kFull, (v >> 62) == 2);
    const int stop = inc ? __ffs(inc) - 1 : 31;
    long long part = lane <= stop ? (long long)(v & kLbVal) : 0;
    excl += warp_sum(part);
    if (inc) break;
    j -= 32;
  }
  if (lane == 0) st_release_u64(&status[t], kLbInc | (unsigned long long)(excl + count));
  return excl;
}

// The two halves of lookback_prefix, for a block that has other work between
// them: one thread publishes the row's count (ticket 0: its inclusive
// prefix) ...
__device__ __forceinline__ void lookback_publish(unsigned long long* status, int64_t t, long long count) {
  st_release_u64(&status[t], (t == 0 ? kLbInc : kLbAgg) | (unsigned long long)count);
}

// ... and later warp 0 sums the counts of all earlier tickets, publishes the
// inclusive prefix and returns the exclusive one (-1 when a wait gave up).
__device__ long long lookback_resolve(unsigned long long* status, int64_t t, long long count) {
  const int lane = threadIdx.x & 31;
  if (t == 0) return 0;
  long long excl = 0;
  int64_t j = t - 1;
  int spins = 0;
  for (;;) {
    const int64_t idx = j - lane;
    const unsigned long long v = idx >= 0 ? ld_acquire_u64(&status[idx]) : kLbInc;
    if (__any_sync(kFull, (v >> 62) == 0)) {
      if (++spins > kLbSpins) return -1;
      __nanosleep(64);
      continue;
    }
    const unsigned inc = __ballot_sync(kFull, (v >> 62) == 2);
    const int stop = inc ? __ffs(inc) - 1 : 31;
    long long part = lane <= stop ? (long long)(v & kLbVal) : 0;
    excl += warp_sum(part);
    if (inc) break;
    j -= 32;
  }
  if (lane == 0) st_release_u64(&status[t], kLbInc | (unsigned long long)(excl + count));
  return excl;
}

__host__ __device__ constexpr int floor_pow2(int x) { return x < 2 ? 1 : 2 * floor_pow2(x / 2); }

template <int BLOCK, int CAP, int NBB, typename VIn, bool FUSED = false>
__global__ void __launch_bounds__(BLOCK)
k_numc_esc_msd(const int32_t* __restrict__ rows, Csr A, Csr B, int32_t b_sorted, const int64_t* __restrict__ crp,
               int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval,
               int32_t* __restrict__ ovf, unsigned int* __restrict__ ovf_count, DevStatus* st, Fused fu) {
  using AT = typename Acc<VIn>::T;
  constexpr int NB = 1 << NBB;
  constexpr int NW = BLOCK / 32;
  constexpr int NG = NB / 32;
  constexpr int NCH = CAP / 32;
  constexpr int ACH = BLOCK < kBChunk ? BLOCK : kBChunk;
  static_assert(kBChunk <= 256, "8-bit A entry indices");
  static_assert(CAP <= 32768 && CAP % 32 == 0, "16-bit counters");
  static_assert(NG <= BLOCK && NCH <= BLOCK && NB % (2 * BLOCK) == 0, "one count per thread in the scans");
  extern __shared__ __align__(16) uint8_t smem[];
  AT* sval = reinterpret_cast<AT*>(smem);
  uint32_t* skey = reinterpret_cast<uint32_t*>(sval + CAP);
  uint32_t* bcnt = skey + CAP;        // NB 16-bit counters
  uint32_t* ccnt = bcnt + NB / 2;     // NCH chunk counts / offsets
  uint8_t* segof = reinterpret_cast<uint8_t*>(ccnt + NCH);
  StageB<VIn>& sg = *reinterpret_cast<StageB<VIn>*>(segof + ((CAP + 15) & ~15));
  __shared__ long long s_tick, s_off;
  int64_t r, tick = 0;
  if (FUSED) {
    if (threadIdx.x == 0) s_tick = (long long)atomicAdd(fu.ticket, 1ull);
    __syncthreads();
    tick = s_tick;
    r = fu.rows[tick];
  } else {
    r = rows[blockIdx.x];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  // fused rows: publish `cnt` and return the row's first position in C (-1
  // when the look-back gave up)
  auto place = [&](long long cnt) -> long long {
    if (warp == 0) {
      const long long ex = lookback_prefix(fu.status, tick, cnt);
      if (lane == 0) {
        s_off = ex < 0 ? -1 : (long long)fu.known[r] + ex;
        fu.row_nz[r] = ex < 0 ? 0 : cnt;
        if (ex < 0) dev_report(st, kDevTimeout, 15, r);
      }
    }
    __syncthreads();
    return s_off;
  };
  // fused rows whose buckets overflow: the distinct count from a hash over the
  // whole shared arena, published so that later rows can go on; the row itself
  // is left to the radix-sort ESC kernel, which writes it at its place
  auto count_and_defer = [&]() {
    constexpr int TS = floor_pow2(CAP * (int)(sizeof(AT) + 4) / 4);
    constexpr int TB = __builtin_ctz(TS);
    uint32_t* tab = reinterpret_cast<uint32_t*>(smem);
    __syncthreads();
    for (int i = threadIdx.x; i < TS; i += BLOCK) tab[i] = kEmptyKey;
    __syncthreads();
    int cnt = 0;
    for (int64_t a0 = as; a0 < ae; a0 += ACH) {
      const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
      const int t = stage_chunk<BLOCK, false, VIn>(A, B, a0, na, sg, segof, CAP, false);
      expand_chunk<BLOCK, false, VIn>(B, t, sg, segof, [&](int32_t key, VIn, VIn, int) {
        uint32_t h = hash_slot((uint32_t)key, TB);
        for (int probe = 0; probe < TS; ++probe) {
          const uint32_t old = atomicCAS(&tab[h], kEmptyKey, (uint32_t)key);
          if (old == kEmptyKey) { ++cnt; return; }
          if (old == (uint32_t)key) return;
          h = (h + 1) & (TS - 1);
        }
      });
      __syncthreads();
    }
    const int distinct = block_sum<BLOCK, int>(cnt, sg.tmp);
    place(distinct);
    if (threadIdx.x == 0) ovf[atomicAdd(ovf_count, 1u)] = (int32_t)r;
  };
  if (threadIdx.x == 0) { sg.kmin = 0xFFFFFFFFu; sg.kmax = 0u; sg.over = 0; }
  for (int i = threadIdx.x; i < NB / 2; i += BLOCK) bcnt[i] = 0u;
  // the column range: from the staged chunk when the row has one chunk,
  // else from a pass over all its A entries (or [0, num_col) when B is unsorted)
  const bool one_chunk = ae - as <= ACH;
  if (!one_chunk) {
    __syncthreads();
    if (b_sorted) {
      uint32_t lo_key = 0xFFFFFFFFu, hi_key = 0u;
      for (int64_t ja = as + threadIdx.x; ja < ae; ja += BLOCK) {
        const int32_t k = A.col[ja];
        const int64_t lo = B.rp[k], hi = B.rp[k + 1];
        if (hi > lo) {
          lo_key = min(lo_key, (uint32_t)__ldg(B.col + lo));
          hi_key = max(hi_key, (uint32_t)__ldg(B.col + hi - 1));
        }
      }
      lo_key = warp_min_u32(lo_key);
      hi_key = warp_max_u32(hi_key);
      if (lane == 0) {
        atomicMin(&sg.kmin, lo_key);
        atomicMax(&sg.kmax, hi_key);
      }
    } else if (threadIdx.x == 0) {
      sg.kmin = 0u;
      sg.kmax = (uint32_t)(B.ncol > 0 ? B.ncol - 1 : 0);
    }
  } else if (!b_sorted && threadIdx.x == 0) {
    sg.kmin = 0u;
    sg.kmax = (uint32_t)(B.ncol > 0 ? B.ncol - 1 : 0);
  }
  __syncthreads();
  // pass 1: keys only, bucket histogram
  int n = 0, total = 0;
  uint32_t lo = 0;
  int shift = 0;
  for (int64_t a0 = as; a0 < ae; a0 += ACH) {
    const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
    total = stage_chunk<BLOCK, true, VIn>(A, B, a0, na, sg, segof, CAP - n, one_chunk && b_sorted);
    if (n + total > CAP) {  // uniform: the bin bound was violated
      if (threadIdx.x == 0) dev_report(st, kDevCapacity, 14, r);
      if (FUSED) place(0);
      return;
    }
    lo = sg.kmin;
    const int bits = (sg.kmax > sg.kmin) ? 32 - __clz(sg.kmax - sg.kmin) : 0;
    shift = bits > NBB ? bits - NBB : 0;
    expand_chunk<BLOCK, false, VIn>(B, total, sg, segof, [&](int32_t key, VIn, VIn, int) {
      bucket_add(bcnt, (int)(((uint32_t)key - lo) >> shift));
    });
    n += total;
    if (!one_chunk) __syncthreads();
  }
  __syncthreads();
  // exclusive scan of the bucket counts: NB / BLOCK consecutive buckets per thread
  constexpr int WPT = NB / (2 * BLOCK);
  {
    uint32_t loc[WPT];
    uint32_t sum = 0, big = 0;
#pragma unroll
    for (int i = 0; i < WPT; ++i) {
      loc[i] = bcnt[threadIdx.x * WPT + i];
      const uint32_t c0 = loc[i] & 0xFFFFu, c1 = loc[i] >> 16;
      sum += c0 + c1;
      big = max(big, max(c0, c1));
    }
    const bool dense_ok = CAP * (int)sizeof(uint8_t) >= kHugeWidth * (int)sizeof(AT) && (1 << shift) <= kHugeWidth;
    if (__syncthreads_or(big > (uint32_t)kBucketLimit && !dense_ok)) {
      if (FUSED) count_and_defer();
      else if (threadIdx.x == 0) ovf[atomicAdd(ovf_count, 1u)] = (int32_t)r;
      return;
    }
    int tot_all;
    uint32_t run = (uint32_t)block_exclusive_sum<BLOCK, int>((int)sum, sg.tmp, tot_all);
#pragma unroll
    for (int i = 0; i < WPT; ++i) {
      const uint32_t c0 = loc[i] & 0xFFFFu, c1 = loc[i] >> 16;
      bcnt[threadIdx.x * WPT + i] = run | ((run + c0) << 16);
      run += c0 + c1;
    }
  }
  __syncthreads();
  // pass 2: (column, a*b) straight into bucket order; bucket b then ends at bucket_get(b)
  if (one_chunk) {
    expand_chunk<BLOCK, true, VIn>(B, total, sg, segof, [&](int32_t key, VIn av, VIn bv, int) {
      const int pos = (int)bucket_add(bcnt, (int)(((uint32_t)key - lo) >> shift));
      skey[pos] = (uint32_t)key;
      sval[pos] = Acc<VIn>::mul(av, bv);
    });
  } else {
    int m = 0;
    for (int64_t a0 = as; a0 < ae; a0 += ACH) {
      const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
      const int t = stage_chunk<BLOCK, true, VIn>(A, B, a0, na, sg, segof, CAP - m, false);
      expand_chunk<BLOCK, true, VIn>(B, t, sg, segof, [&](int32_t key, VIn av, VIn bv, int) {
        const int pos = (int)bucket_add(bcnt, (int)(((uint32_t)key - lo) >> shift));
        skey[pos] = (uint32_t)key;
        sval[pos] = Acc<VIn>::mul(av, bv);
      });
      m += t;
      __syncthreads();
    }
  }
  __syncthreads();
  // sort each bucket, sum equal columns, compact them to the bucket front:
  // one lane per bucket of at most 8 pairs; the warp then takes its larger
  // buckets (about 1 in 100, and the diagonal column's) one at a time, so
  // they overlap the other warps' small buckets.  Buckets of more than
  // kBucketLimit pairs are queued for the whole block.
  __shared__ uint16_t s_huge[kHugeBuckets];
  __shared__ int s_nhuge;
  if (threadIdx.x == 0) s_nhuge = 0;
  __syncthreads();
  for (int g = warp; g < NG; g += NW) {
    const int b = g * 32 + lane;
    const int s = b ? (int)bucket_get(bcnt, b - 1) : 0, e = (int)bucket_get(bcnt, b);
    if (e - s > kBucketLimit) {
      const int slot = atomicAdd(&s_nhuge, 1);
      if (slot < kHugeBuckets) s_huge[slot] = (uint16_t)b;
    }
    // one network size for the whole warp: the smallest that fits its
    // largest bucket of at most 8 pairs
    const int small = (e - s <= 8) ? e - s : 0;
    const int mx = __reduce_max_sync(kFull, small);
    if (small > 0) {
      const uint32_t kbase = lo + ((uint32_t)b << shift);
      if (mx <= 4) sort_compact_small<4, AT>(skey, sval, s, e, kbase);
      else if (mx <= 6) sort_compact_small<6, AT>(skey, sval, s, e, kbase);
      else sort_compact_small<8, AT>(skey, sval, s, e, kbase);
    }
    for (unsigned big = __ballot_sync(kFull, e - s > 8 && e - s <= kBucketLimit); big; big &= big - 1) {
      const int l = __ffs(big) - 1;
      warp_sort_compact<AT>(skey, sval, __shfl_sync(kFull, s, l), __shfl_sync(kFull, e, l));
    }
  }
  __syncthreads();
  if (s_nhuge > kHugeBuckets) {  // uniform: too many huge buckets for this form
    if (FUSED) count_and_defer();
    else if (threadIdx.x == 0) ovf[atomicAdd(ovf_count, 1u)] = (int32_t)r;
    return;
  }
  if (s_nhuge > 0) {
    // the whole block, one huge bucket at a time: sums by column offset in a
    // dense array over the byte table, then the present columns in order
    __shared__ uint32_t s_hmask[kHugeWidth / 32];
    __shared__ int s_hpre[kHugeWidth / 32];
    AT* dacc = reinterpret_cast<AT*>(segof);
    const int width = 1 << shift;
    for (int h = 0; h < s_nhuge; ++h) {
      const int b = s_huge[h];
      const int s = b ? (int)bucket_get(bcnt, b - 1) : 0, e = (int)bucket_get(bcnt, b);
      const uint32_t kb = lo + ((uint32_t)b << shift);
      __syncthreads();
      for (int j = threadIdx.x; j < width; j += BLOCK) dacc[j] = AT(0);
      if (threadIdx.x < kHugeWidth / 32) s_hmask[threadIdx.x] = 0u;
      __syncthreads();
      for (int i = s + threadIdx.x; i < e; i += BLOCK) {
        const int off = (int)(skey[i] - kb);
        atomic_add_sh(&dacc[off], sval[i]);
        atomicOr(&s_hmask[off >> 5], 1u << (off & 31));
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kHugeWidth / 32; ++w) {
          s_hpre[w] = run;
          run += __popc(s_hmask[w]);
        }
      }
      __syncthreads();
      const int heads = s_hpre[kHugeWidth / 32 - 1] + __popc(s_hmask[kHugeWidth / 32 - 1]);
      for (int j = threadIdx.x; j < width; j += BLOCK) {
        const uint32_t m = s_hmask[j >> 5];
        if (m & (1u << (j & 31))) {
          const int pos = s + s_hpre[j >> 5] + __popc(m & ((1u << (j & 31)) - 1u));
          skey[pos] = kb + (uint32_t)j;
          sval[pos] = dacc[j];
        }
      }
      for (int i = s + heads + threadIdx.x; i < e; i += BLOCK) skey[i] = kEmptyKey;
    }
  }
  __syncthreads();
  // distinct pairs per 32-slot chunk, then chunk offsets
  const int nch = (n + 31) >> 5;
  for (int c = warp; c < nch; c += NW) {
    const int t = c * 32 + lane;
    const bool valid = t < n && skey[t] != kEmptyKey;
    const unsigned m = __ballot_sync(kFull, valid);
    if (lane == 0) ccnt[c] = __popc(m);
  }
  __syncthreads();
  int distinct;
  {
    const int cnum = threadIdx.x < nch ? (int)ccnt[threadIdx.x] : 0;
    const int ex = block_exclusive_sum<BLOCK, int>(cnum, sg.tmp, distinct);
    if (threadIdx.x < nch) ccnt[threadIdx.x] = (uint32_t)ex;
  }
  __syncthreads();
  int64_t c0, nz;
  if (FUSED) {
    c0 = place(distinct);
    if (c0 < 0) return;
    nz = distinct;
    if (c0 + nz > fu.cap) {
      if (threadIdx.x == 0) dev_report(st, kDevRowOverflow, 15, r);
      return;
    }
  } else {
    c0 = crp[r];
    nz = crp[r + 1] - c0;
  }
  for (int c = warp; c < nch; c += NW) {
    const int t = c * 32 + lane;
    uint32_t key = kEmptyKey;
    if (t < n) key = skey[t];
    const bool valid = key != kEmptyKey;
    const unsigned m = __ballot_sync(kFull, valid);
    if (valid) {
      const int64_t pos = (int64_t)ccnt[c] + __popc(m & lanemask_lt());
      if (pos < nz) {
        ccol[c0 + pos] = (int32_t)key;
        cval[c0 + pos] = sval[t];
      }
    }
  }
  if (!FUSED && threadIdx.x == 0 && distinct != nz)
    dev_report(st, distinct > nz ? kDevRowOverflow : kDevRowUnderflow, 14, r);
}

// ---- index form of the bucketed ESC kernel ---------------------------------
// For rows whose A entries fit one staged chunk (at most kBChunk).  Shared
// memory holds each product's column (4 bytes), its product index (2 bytes)
// and later its place in the row (2 bytes) instead of its column and value
// (12 bytes), so more rows are resident per SM; the kernel is bound by load
// and barrier latency, which more resident rows hide.  The steps are those
// of k_numc_esc_msd (ams_hsersc_numc_krnl, src/ams/ams_utils.c:399-456): a
// keys-only histogram into 2^NBB buckets, a second keys-only expansion that
// scatters (column, product index) into bucket order, and a sort of each
// bucket: a network per lane for buckets of up to 8, a warp rank sort for up
// to kBucketLimit, and a dense sum by the whole block for one bucket of more
// over at most kHugeWidth columns.  Equal columns stay side by side.  A pass
// in sorted order writes each distinct column to C and records, for every
// product, the place of its column in the row; a last pass in product order
// loads the B values (whole sectors, as the B rows lie in memory) and stores
// each product a_ik * b_kj at its place, with a global atomic add where
// several products share a column (the place is zeroed first).  A row with
// more A entries than one chunk, with two or more buckets of more than
// kBucketLimit products, or with one that spans more than kHugeWidth
// columns, is counted with a shared-memory hash and left to the radix-sort
// ESC kernel (appended to `ovf`), as in k_numc_esc_msd.
constexpr int kIdxMinBlocks = 4;

// Values of the staged chunk's products only (no columns): f(a, b, p).
template <int BLOCK, typename VIn, typename F>
__device__ __forceinline__ void expand_values(const Csr& B, int total, const StageB<VIn>& sg,
                                              const uint8_t* __restrict__ segof, F&& f) {
  const VIn* __restrict__ bval = static_cast<const VIn*>(B.val);
  for (int p0 = threadIdx.x; p0 < total; p0 += BLOCK * kUnroll) {
    VIn bv[kUnroll];
    int sgi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int p = p0 + u * BLOCK;
      sgi[u] = -1;
      if (p < total) {
        const int s = segof[p];
        bv[u] = __ldg(bval + sg.bs[s] + (p - sg.pre[s]));
        sgi[u] = s;
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (sgi[u] >= 0) f(sg.av[sgi[u]], bv[u], p0 + u * BLOCK);
  }
}

// The same values, a warp per B row (segment) of the staged chunk: the
// segment's start, first product and A value are read once per warp, and
// the lanes load the row's values with consecutive addresses.  Two segments
// are in flight per warp.  Suits chunks whose B rows are long (the lanes of a
// short row idle); f(a, b, p) as in expand_values.
template <int BLOCK, typename VIn, typename F>
__device__ __forceinline__ void expand_values_seg(const Csr& B, int na, const StageB<VIn>& sg, F&& f) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const VIn* __restrict__ bval = static_cast<const VIn*>(B.val);
  for (int s0 = warp; s0 < na; s0 += 2 * NW) {
    const int s1 = s0 + NW;
    const int b0 = sg.pre[s0], l0 = sg.pre[s0 + 1] - b0;
    const int b1 = s1 < na ? sg.pre[s1] : 0, l1 = s1 < na ? sg.pre[s1 + 1] - b1 : 0;
    const VIn a0 = sg.av[s0], a1 = s1 < na ? sg.av[s1] : VIn(0);
    const VIn* __restrict__ r0 = bval + sg.bs[s0];
    const VIn* __restrict__ r1 = bval + (s1 < na ? sg.bs[s1] : 0);
    const int lmax = l0 > l1 ? l0 : l1;
    for (int i = lane; i < lmax; i += 64) {
      const int j = i + 32;
      VIn v[4];
      v[0] = i < l0 ? __ldg(r0 + i) : VIn(0);
      v[1] = j < l0 ? __ldg(r0 + j) : VIn(0);
      v[2] = i < l1 ? __ldg(r1 + i) : VIn(0);
      v[3] = j < l1 ? __ldg(r1 + j) : VIn(0);
      if (i < l0) f(a0, v[0], b0 + i);
      if (j < l0) f(a0, v[1], b0 + j);
      if (i < l1) f(a1, v[2], b1 + i);
      if (j < l1) f(a1, v[3], b1 + j);
    }
  }
}

template <int N>
__device__ __forceinline__ void sort_perm_small(uint32_t* __restrict__ skey, uint16_t* __restrict__ sidx, int s, int e,
                                                uint32_t kbase) {
  const int nb = e - s;
  uint32_t w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) w[i] = i < nb ? sortnet_pack(skey[s + i] - kbase, i) : 0xFFFFFFFFu;
  sort_net(w);
  uint16_t q[N];
#pragma unroll
  for (int i = 0; i < N; ++i) q[i] = i < nb ? sidx[s + sortnet_slot(w[i])] : uint16_t(0);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    if (i < nb) {
      skey[s + i] = kbase + sortnet_offset(w[i]);
      sidx[s + i] = q[i];
    }
  }
}

// Whole-warp stable rank sort of one bucket [s, e), e - s <= 128, of
// (column, product index) pairs.
__device__ __forceinline__ void warp_sort_perm(uint32_t* __restrict__ skey, uint16_t* __restrict__ sidx, int s, int e) {
  constexpr int PER = 4;
  const int lane = threadIdx.x & 31;
  const int b = e - s;
  uint32_t k[PER];
  uint16_t q[PER];
  int rk[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int t = lane + 32 * i;
    k[i] = t < b ? skey[s + t] : kEmptyKey;
    q[i] = t < b ? sidx[s + t] : uint16_t(0);
    rk[i] = 0;
  }
#pragma unroll 4
  for (int j = 0; j < b; ++j) {
    const uint32_t kj = skey[s + j];
#pragma unroll
    for (int i = 0; i < PER; ++i) rk[i] += (kj < k[i]) || (kj == k[i] && j < lane + 32 * i);
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    if (lane + 32 * i < b) {
      skey[s + rk[i]] = k[i];
      sidx[s + rk[i]] = q[i];
    }
  }
  __syncwarp();
}

template <int BLOCK, int CAP, int NBB, typename VIn, bool FUSED = false, bool REGK = false>
__global__ void __launch_bounds__(BLOCK, kIdxMinBlocks)
k_numc_esc_idx(const int32_t* __restrict__ rows, Csr A, Csr B, int32_t b_sorted, const int64_t* __restrict__ crp,
               int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval,
               int32_t* __restrict__ ovf, unsigned int* __restrict__ ovf_count, DevStatus* st, Fused fu) {
  using AT = typename Acc<VIn>::T;
  constexpr int NB = 1 << NBB;
  constexpr int NW = BLOCK / 32;
  constexpr int NG = NB / 32;
  constexpr int NCH = CAP / 32;
  constexpr int NCHP = (NCH + 3) & ~3;  // chunk counts padded to 16 bytes
  constexpr int ACH = BLOCK < kBChunk ? BLOCK : kBChunk;
  // the hash of deferred rows spans columns, indices, places, bucket counts, chunk counts and masks
  constexpr int TS = floor_pow2((CAP * 8 + NB * 2 + NCHP * 8) / 4);
  constexpr int TB = __builtin_ctz(TS);
  static_assert(CAP < 32768 && CAP % 32 == 0, "16-bit counters, product indices and places");
  static_assert(NG <= BLOCK && NCH <= BLOCK && NB % (2 * BLOCK) == 0, "one count per thread in the scans");
  static_assert(TS >= CAP + CAP / 4, "hash of deferred rows: load at most 0.8");
  extern __shared__ __align__(16) uint8_t smem[];
  // REGK puts place_of first: everything after it up to the byte table
  // (and the byte table too, when the value pass walks B rows) is dead by
  // the value pass and then holds the row's values at their places
  uint16_t* place_of = REGK ? reinterpret_cast<uint16_t*>(smem)
                            : reinterpret_cast<uint16_t*>(smem + size_t(CAP) * 6);  // per product: its column's place
  uint32_t* skey = reinterpret_cast<uint32_t*>(REGK ? smem + size_t(CAP) * 2 : smem);
  uint16_t* sidx = reinterpret_cast<uint16_t*>(skey + CAP);
  uint32_t* bcnt = reinterpret_cast<uint32_t*>(smem + size_t(CAP) * 8);  // NB 16-bit counters
  uint32_t* ccnt = bcnt + NB / 2;                              // NCH head counts / offsets
  uint32_t* hmw = ccnt + NCHP;                                 // NCH head masks
  uint8_t* segof = reinterpret_cast<uint8_t*>(hmw + NCHP);
  StageB<VIn>& sg = *reinterpret_cast<StageB<VIn>*>(segof + ((CAP + 15) & ~15));
  static_assert(CAP % 32 == 0, "8-byte alignment of the staged values after place_of");
  __shared__ long long s_tick, s_off;
  __shared__ int s_huge, s_hlast;
  __shared__ uint32_t s_hkb;       // first column of the huge bucket
  __shared__ AT hsum[kHugeWidth];  // the huge bucket's sums by column offset
  __shared__ uint32_t hmask[kHugeWidth / 32];
  __shared__ int hpre[kHugeWidth / 32 + 1];
  constexpr uint16_t kFromSum = 0xFFFE, kNoProduct = 0xFFFF;
  static_assert(CAP < kFromSum, "product indices below the markers");
  // place_of: bit 15 set when the column has several products (atomic add);
  // kSkip for products of the huge bucket, summed in hsum
  constexpr uint16_t kShared = 0x8000, kSkip = 0xFFFF;
  // a_ik * b_kj of product p of the staged chunk (0 for a filler slot)
  auto slot_value = [&](uint16_t p) -> AT {
    if (p == kNoProduct) return AT(0);
    const int sgi = segof[p];
    return Acc<VIn>::mul(sg.av[sgi], __ldg(static_cast<const VIn*>(B.val) + sg.bs[sgi] + ((int)p - sg.pre[sgi])));
  };
  int64_t r, tick = 0;
  if (FUSED) {
    if (threadIdx.x == 0) s_tick = (long long)atomicAdd(fu.ticket, 1ull);
    __syncthreads();
    tick = s_tick;
    r = fu.rows[tick];
  } else {
    r = rows[blockIdx.x];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  // fused rows: publish `cnt` and return the row's first position in C (-1
  // when the look-back gave up)
  auto place = [&](long long cnt) -> long long {
    if (warp == 0) {
      const long long ex = lookback_prefix(fu.status, tick, cnt);
      if (lane == 0) {
        s_off = ex < 0 ? -1 : (long long)fu.known[r] + ex;
        fu.row_nz[r] = ex < 0 ? 0 : cnt;
        if (ex < 0) dev_report(st, kDevTimeout, 16, r);
      }
    }
    __syncthreads();
    return s_off;
  };
  // rows this form does not take: fused ones are counted here (a hash over
  // the shared arena) and published; all go to the radix-sort ESC kernel
  auto defer = [&]() {
    if (FUSED) {
      uint32_t* tab = reinterpret_cast<uint32_t*>(smem);
      __syncthreads();
      for (int i = threadIdx.x; i < TS; i += BLOCK) tab[i] = kEmptyKey;
      __syncthreads();
      int cnt = 0;
      for (int64_t a0 = as; a0 < ae; a0 += ACH) {
        const int na = (int)((ae - a0) < (int64_t)ACH ? (ae - a0) : (int64_t)ACH);
        const int t = stage_chunk<BLOCK, false, VIn>(A, B, a0, na, sg, segof, CAP, false);
        expand_chunk<BLOCK, false, VIn>(B, t, sg, segof, [&](int32_t key, VIn, VIn, int) {
          uint32_t h = hash_slot((uint32_t)key, TB);
          for (int probe = 0; probe < TS; ++probe) {
            const uint32_t old = atomicCAS(&tab[h], kEmptyKey, (uint32_t)key);
            if (old == kEmptyKey) { ++cnt; return; }
            if (old == (uint32_t)key) return;
            h = (h + 1) & (TS - 1);
          }
        });
        __syncthreads();
      }
      place(block_sum<BLOCK, int>(cnt, sg.tmp));
    }
    if (threadIdx.x == 0) ovf[atomicAdd(ovf_count, 1u)] = (int32_t)r;
  };
  if (ae - as > ACH) {  // uniform: more than one staged chunk
    defer();
    return;
  }
  if (threadIdx.x == 0) {
    sg.kmin = b_sorted ? 0xFFFFFFFFu : 0u;
    sg.kmax = b_sorted ? 0u : (uint32_t)(B.ncol > 0 ? B.ncol - 1 : 0);
    sg.over = 0;
  }
  for (int i = threadIdx.x; i < NB / 2; i += BLOCK) bcnt[i] = 0u;
  __syncthreads();
  const int n = stage_chunk<BLOCK, true, VIn>(A, B, as, (int)(ae - as), sg, segof, CAP, b_sorted != 0);
  if (n > CAP) {  // uniform: the bin bound was violated
    if (threadIdx.x == 0) dev_report(st, kDevCapacity, 16, r);
    if (FUSED) place(0);
    return;
  }
  const uint32_t lo = sg.kmin;
  const int bits = (sg.kmax > sg.kmin) ? 32 - __clz(sg.kmax - sg.kmin) : 0;
  const int shift = bits > NBB ? bits - NBB : 0;
  // pass 1: keys only, bucket histogram.  REGK: the thread's keys (products
  // threadIdx.x + u * BLOCK) stay in registers for pass 2, so B's columns
  // are read once
  int huge;
  constexpr int NPT = REGK ? (CAP + BLOCK - 1) / BLOCK : 1;
  uint32_t rkey[NPT];
  if constexpr (REGK) {
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
      const int p = threadIdx.x + u * BLOCK;
      if (p < n) {
        const int sgi = segof[p];
        rkey[u] = (uint32_t)__ldg(B.col + sg.bs[sgi] + (p - sg.pre[sgi]));
      }
    }
#pragma unroll
    for (int u = 0; u < NPT; ++u)
      if (threadIdx.x + u * BLOCK < n) bucket_add(bcnt, (int)((rkey[u] - lo) >> shift));
  } else {
    expand_chunk<BLOCK, false, VIn>(B, n, sg, segof, [&](int32_t key, VIn, VIn, int) {
      bucket_add(bcnt, (int)(((uint32_t)key - lo) >> shift));
    });
  }
  __syncthreads();
  // exclusive scan of the bucket counts: NB / BLOCK consecutive buckets per thread
  constexpr int WPT = NB / (2 * BLOCK);
  {
    uint32_t loc[WPT];
    uint32_t sum = 0;
    int nh = 0;  // buckets of more than kBucketLimit pairs
#pragma unroll
    for (int i = 0; i < WPT; ++i) {
      loc[i] = bcnt[threadIdx.x * WPT + i];
      const uint32_t c0 = loc[i] & 0xFFFFu, c1 = loc[i] >> 16;
      sum += c0 + c1;
      nh += (c0 > (uint32_t)kBucketLimit) + (c1 > (uint32_t)kBucketLimit);
    }
    // at most one huge bucket, over at most kHugeWidth columns, in this form
    huge = __syncthreads_count(nh > 0);
    if (__syncthreads_or(nh > 1 || (nh > 0 && (1 << shift) > kHugeWidth)) || huge > 1) {
      defer();
      return;
    }
    int tot_all;
    uint32_t run = (uint32_t)block_exclusive_sum<BLOCK, int>((int)sum, sg.tmp, tot_all);
#pragma unroll
    for (int i = 0; i < WPT; ++i) {
      const uint32_t c0 = loc[i] & 0xFFFFu, c1 = loc[i] >> 16;
      bcnt[threadIdx.x * WPT + i] = run | ((run + c0) << 16);
      run += c0 + c1;
    }
  }
  __syncthreads();
  // pass 2: (column, product index) into bucket order
  if constexpr (REGK) {
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
      const int p = threadIdx.x + u * BLOCK;
      if (p < n) {
        const int pos = (int)bucket_add(bcnt, (int)((rkey[u] - lo) >> shift));
        skey[pos] = rkey[u];
        sidx[pos] = (uint16_t)p;
      }
    }
  } else {
    expand_chunk<BLOCK, false, VIn>(B, n, sg, segof, [&](int32_t key, VIn, VIn, int p) {
      const int pos = (int)bucket_add(bcnt, (int)(((uint32_t)key - lo) >> shift));
      skey[pos] = (uint32_t)key;
      sidx[pos] = (uint16_t)p;
    });
  }
  __syncthreads();
  // sort each bucket: a lane per bucket of 2..8 pairs (one network size per
  // warp), then the warp's buckets of 9..kBucketLimit pairs one at a time;
  // a bucket of more pairs over at most kHugeWidth columns (hub columns) is
  // left to the whole block
  for (int g = warp; g < NG; g += NW) {
    const int b = g * 32 + lane;
    const int s = b ? (int)bucket_get(bcnt, b - 1) : 0, e = (int)bucket_get(bcnt, b);
    if (e - s > kBucketLimit) s_huge = b;
    const int small = (e - s <= 8) ? e - s : 0;
    const int mx = __reduce_max_sync(kFull, small);
    if (small > 1) {
      const uint32_t kbase = lo + ((uint32_t)b << shift);
      if (mx <= 4) sort_perm_small<4>(skey, sidx, s, e, kbase);
      else if (mx <= 6) sort_perm_small<6>(skey, sidx, s, e, kbase);
      else sort_perm_small<8>(skey, sidx, s, e, kbase);
    }
    for (unsigned bigm = __ballot_sync(kFull, e - s > 8 && e - s <= kBucketLimit); bigm; bigm &= bigm - 1) {
      const int l = __ffs(bigm) - 1;
      warp_sort_perm(skey, sidx, __shfl_sync(kFull, s, l), __shfl_sync(kFull, e, l));
    }
  }
  __syncthreads();
  if (huge) {
    // sums by column offset in hsum, then the bucket's slots become its
    // present columns in order (product index kFromSum: the value is the
    // sum) followed by fillers repeating the last column (kNoProduct: no
    // value), so the runs and heads below see one slot per column
    const int b = s_huge;
    const int s = b ? (int)bucket_get(bcnt, b - 1) : 0, e = (int)bucket_get(bcnt, b);
    const int width = 1 << shift;
    const uint32_t kb = lo + ((uint32_t)b << shift);
    for (int j = threadIdx.x; j < width; j += BLOCK) hsum[j] = AT(0);
    if (threadIdx.x < kHugeWidth / 32) hmask[threadIdx.x] = 0u;
    if (threadIdx.x == 0) s_hkb = kb;
    __syncthreads();
    for (int i = s + threadIdx.x; i < e; i += BLOCK) {
      const int off = (int)(skey[i] - kb);
      atomic_add_sh(&hsum[off], slot_value(sidx[i]));
      atomicOr(&hmask[off >> 5], 1u << (off & 31));
      place_of[sidx[i]] = kSkip;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0, lastc = 0;
      for (int w = 0; w < kHugeWidth / 32; ++w) {
        hpre[w] = run;
        run += __popc(hmask[w]);
        if (hmask[w]) lastc = w * 32 + 31 - __clz(hmask[w]);
      }
      hpre[kHugeWidth / 32] = run;
      s_hlast = lastc;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < width; j += BLOCK) {
      const uint32_t m = hmask[j >> 5];
      if (m & (1u << (j & 31))) {
        const int pos = s + hpre[j >> 5] + __popc(m & ((1u << (j & 31)) - 1u));
        skey[pos] = kb + (uint32_t)j;
        sidx[pos] = kFromSum;
      }
    }
    for (int i = s + hpre[kHugeWidth / 32] + threadIdx.x; i < e; i += BLOCK) {
      skey[i] = kb + (uint32_t)s_hlast;
      sidx[i] = kNoProduct;
    }
    __syncthreads();
  }
  // run heads (first slot of each column) per 32-slot chunk, then offsets
  const int nch = (n + 31) >> 5;
  auto is_head = [&](int t) { return t < n && (t == 0 || skey[t] != skey[t - 1]); };
  for (int c = warp; c < nch; c += NW) {
    const unsigned m = __ballot_sync(kFull, is_head(c * 32 + lane));
    if (lane == 0) {
      ccnt[c] = __popc(m);
      hmw[c] = m;
    }
  }
  __syncthreads();
  int distinct;
  {
    const int cnum = threadIdx.x < nch ? (int)ccnt[threadIdx.x] : 0;
    const int ex = block_exclusive_sum<BLOCK, int>(cnum, sg.tmp, distinct);
    if (threadIdx.x < nch) ccnt[threadIdx.x] = (uint32_t)ex;
  }
  __syncthreads();
  // fused rows: the count goes out now, the look-back waits until the
  // places below are recorded, so the wait for earlier rows overlaps them
  if (FUSED && threadIdx.x == 0) lookback_publish(fu.status, tick, distinct);
  const int64_t nz = FUSED ? (int64_t)distinct : crp[r + 1] - crp[r];
  auto head_at = [&](int t) -> bool { return t < n && ((hmw[t >> 5] >> (t & 31)) & 1u); };
  // each product's place: the run of its column, flagged when the run has
  // several products (those add into C atomically)
  for (int c = warp; c < nch; c += NW) {
    const int t = c * 32 + lane;
    const unsigned m = hmw[c];
    if (t < n) {
      const uint16_t p = sidx[t];
      const int run = (int)ccnt[c] + __popc(m & ((lanemask_lt() << 1) | 1u)) - 1;
      if (p < kFromSum) {
        const bool single = ((m >> lane) & 1u) && (t + 1 == n || head_at(t + 1));
        place_of[p] = run >= nz ? kSkip : (uint16_t)run | (single ? 0 : kShared);
      }
    }
  }
  int64_t c0;
  if (FUSED) {
    if (warp == 0) {
      const long long ex = lookback_resolve(fu.status, tick, distinct);
      if (lane == 0) {
        s_off = ex < 0 ? -1 : (long long)fu.known[r] + ex;
        fu.row_nz[r] = ex < 0 ? 0 : distinct;
        if (ex < 0) dev_report(st, kDevTimeout, 16, r);
      }
    }
    __syncthreads();
    c0 = s_off;
    if (c0 < 0) return;
    if (c0 + nz > fu.cap) {
      if (threadIdx.x == 0) dev_report(st, kDevRowOverflow, 16, r);
      return;
    }
  } else {
    c0 = crp[r];
    __syncthreads();
  }
  // REGK: values staged in shared memory at their places and copied out in
  // order, when they fit the dead part of the arena (with the byte table
  // when the value pass walks B rows)
  const bool seg_walk = REGK && n >= 32 * (int)(ae - as) && (int)(ae - as) >= 2 * NW;
  const size_t dead = size_t(CAP) * 6 + size_t(NB) * 2 + size_t(NCHP) * 8 + (seg_walk ? ((CAP + 15) & ~15) : 0);
  const bool stage = REGK && (size_t)nz * sizeof(AT) <= dead;
  AT* sval = reinterpret_cast<AT*>(skey);
  if (stage && threadIdx.x == 0) s_hlast = 0x7FFFFFFF;  // reused: the huge bucket's first place
  __syncthreads();
  // sorted order: each distinct column to C; the huge bucket's sums; a zero
  // where several products will add (staged values are zeroed below)
  for (int c = warp; c < nch; c += NW) {
    const int t = c * 32 + lane;
    const unsigned m = hmw[c];
    if ((m >> lane) & 1u) {
      const int run = (int)ccnt[c] + __popc(m & lanemask_lt());
      if (run < nz) {
        const uint32_t key = skey[t];
        ccol[c0 + run] = (int32_t)key;
        if (sidx[t] == kFromSum) {
          cval[c0 + run] = hsum[key - s_hkb];
          if (stage) atomicMin(&s_hlast, run);
        } else if (!stage && t + 1 < n && !head_at(t + 1) && sidx[t + 1] != kNoProduct) {
          cval[c0 + run] = AT(0);
        }
      }
    }
  }
  __syncthreads();
  int hp0 = 0, hp1 = 0;  // places of the huge bucket's columns, written above from its sums
  if (stage) {
    if (huge) {
      hp0 = s_hlast;
      hp1 = hp0 + hpre[kHugeWidth / 32];
    }
    for (int i = threadIdx.x; i < (int)nz; i += BLOCK) sval[i] = AT(0);
    __syncthreads();
  }
  // product order: a_ik * b_kj to its place (REGK: a warp per B row when
  // the chunk's B rows average at least 32 products and there are at least
  // two per warp; a row of a few long B rows, as in R-MAT G500 and Zipf
  // products, would leave most warps idle that way)
  auto put = [&](VIn av, VIn bv, int p) {
    const uint16_t o = place_of[p];
    if (o == kSkip) return;
    const AT v = Acc<VIn>::mul(av, bv);
    if (o & kShared) Acc<VIn>::atomic_add(&cval[c0 + (o & ~kShared)], v);
    else cval[c0 + o] = v;
  };
  auto put_staged = [&](VIn av, VIn bv, int p) {
    const uint16_t o = place_of[p];
    if (o == kSkip) return;
    const AT v = Acc<VIn>::mul(av, bv);
    if (o & kShared) atomic_add_sh(&sval[o & ~kShared], v);
    else sval[o] = v;
  };
  if (stage) {
    if (seg_walk) expand_values_seg<BLOCK, VIn>(B, (int)(ae - as), sg, put_staged);
    else expand_values<BLOCK, VIn>(B, n, sg, segof, put_staged);
    __syncthreads();
    for (int i = threadIdx.x; i < (int)nz; i += BLOCK)
      if (i < hp0 || i >= hp1) cval[c0 + i] = sval[i];
  } else if (seg_walk) {
    expand_values_seg<BLOCK, VIn>(B, (int)(ae - as), sg, put);
  } else {
    expand_values<BLOCK, VIn>(B, n, sg, segof, put);
  }
  if (!FUSED && threadIdx.x == 0 && distinct != nz)
    dev_report(st, distinct > nz ? kDevRowOverflow : kDevRowUnderflow, 16, r);
}

// Hash accumulator for rows with at most 2^TBITS / 2 distinct columns: linear
// probing on 32-bit keys with the value summed by shared-memory atomics
// (ams_hash_numc_krnl, src/ams/ams_utils.c:238-296, in shared memory), then
// the occupied slots are compacted, sorted by column, and written in order.
template <int BLOCK, int TBITS, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_numc_hash(const int32_t* __restrict__ rows, Csr A, Csr B, const int64_t* __restrict__ crp,
            int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval, DevStatus* st) {
  using AT = typename Acc<VIn>::T;
  constexpr int T = 1 << TBITS;
  constexpr int NCAP = T / 2;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* tkey = reinterpret_cast<uint32_t*>(smem);         // T keys; later NCAP sort items
  AT* tval = reinterpret_cast<AT*>(smem + T * sizeof(uint32_t));
  uint64_t* items = reinterpret_cast<uint64_t*>(tval + T);     // NCAP compacted items
  SortScratch<BLOCK>& ss = *reinterpret_cast<SortScratch<BLOCK>*>(items + NCAP);
  Stage<VIn>& sg = *reinterpret_cast<Stage<VIn>*>(reinterpret_cast<uint8_t*>(&ss) + sizeof(SortScratch<BLOCK>));
  __shared__ uint32_t s_min, s_max;
  __shared__ int s_cnt, s_full;
  const int64_t r = rows[blockIdx.x];
  for (int i = threadIdx.x; i < T; i += BLOCK) {
    tkey[i] = kEmptyKey;
    tval[i] = AT(0);
  }
  if (threadIdx.x == 0) { s_min = 0xFFFFFFFFu; s_max = 0u; s_cnt = 0; s_full = 0; }
  __syncthreads();
  bool full = false;
  expand_row<BLOCK, true, VIn>(A, B, r, sg, false, 0, 0, [&](int32_t key, VIn av, VIn bv, int64_t) {
    const AT v = Acc<VIn>::mul(av, bv);
    uint32_t h = hash_slot((uint32_t)key, TBITS);
    for (int probe = 0; probe < T; ++probe) {
      const uint32_t cur = tkey[h];
      if (cur == (uint32_t)key) { Acc<VIn>::atomic_add(&tval[h], v); return; }
      if (cur == kEmptyKey) {
        const uint32_t old = atomicCAS(&tkey[h], kEmptyKey, (uint32_t)key);
        if (old == kEmptyKey || old == (uint32_t)key) { Acc<VIn>::atomic_add(&tval[h], v); return; }
      }
      h = (h + 1) & (T - 1);
    }
    full = true;
  });
  if (full) s_full = 1;
  __syncthreads();
  // compact occupied slots into items (warp-aggregated slot reservation)
  const int lane = threadIdx.x & 31;
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u;
  for (int i0 = 0; i0 < T; i0 += BLOCK) {
    const int i = i0 + threadIdx.x;
    const uint32_t k = i < T ? tkey[i] : kEmptyKey;
    const bool occ = k != kEmptyKey;
    const unsigned m = __ballot_sync(kFull, occ);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(&s_cnt, __popc(m));
    base = __shfl_sync(kFull, base, 0);
    if (occ) {
      const int pos = base + __popc(m & lanemask_lt());
      if (pos < NCAP) items[pos] = ((uint64_t)k << 32) | (uint64_t)i;
      kmin = min(kmin, k);
      kmax = max(kmax, k);
    }
  }
  kmin = warp_min_u32(kmin);
  kmax = warp_max_u32(kmax);
  if (lane == 0) {
    atomicMin(&s_min, kmin);
    atomicMax(&s_max, kmax);
  }
  __syncthreads();
  const int64_t c0 = crp[r], nz = crp[r + 1] - c0;
  const int n = s_cnt;
  if (s_full || n > NCAP) {
    if (threadIdx.x == 0) dev_report(st, kDevTableFull, 12, r);
    return;
  }
  uint64_t* spare = reinterpret_cast<uint64_t*>(tkey);  // keys are no longer needed
  const uint64_t* sorted = block_radix_sort<BLOCK>(items, spare, n, s_min, s_max, ss.hist, ss.tmp);
  for (int t = threadIdx.x; t < n && t < nz; t += BLOCK) {
    const uint64_t it = sorted[t];
    ccol[c0 + t] = (int32_t)(it >> 32);
    cval[c0 + t] = tval[(uint32_t)it];
  }
  if (threadIdx.x == 0 && n != nz) dev_report(st, n > nz ? kDevRowOverflow : kDevRowUnderflow, 12, r);
}

// Heavy rows in one pass per slice of kRankCols columns of the row's column
// range: a keys-only expansion marks the row's columns in a shared-memory
// bitmap (or the symbolic kernel's kept bitmap is loaded), the rank of every
// column comes from a 32-bit base per group of 8 words plus a 16-bit rank of
// each word within its group, the column indices are written to C from the
// bitmap and the values zeroed, and a second expansion adds every product
// straight into its place in C with a global atomic add (resolved in L2: a
// row's values are at most 8 bytes x nnz(row) there).  A range wider than one
// slice is cut into slices, B rows cut to each by binary search (B rows
// sorted).
template <int BLOCK, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_numc_dense(const int32_t* __restrict__ rows, Csr A, Csr B, int64_t c_ncol, int32_t b_sorted,
             const int64_t* __restrict__ crp, int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval,
             const uint32_t* __restrict__ saved, const int32_t* __restrict__ saved_slot, int saved_slices,
             DevStatus* st) {
  using AT = typename Acc<VIn>::T;
  constexpr int NWORD = kRankCols / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem);
  uint32_t* gbase = bm + NWORD;                                       // NWORD / 8 group bases
  uint16_t* wrank = reinterpret_cast<uint16_t*>(gbase + NWORD / 8);   // NWORD ranks within the group
  Stage<VIn>& sg = *reinterpret_cast<Stage<VIn>*>(reinterpret_cast<uint8_t*>(wrank + NWORD));
  const int64_t r = rows[blockIdx.x];
  const int64_t c0r = crp[r], nz = crp[r + 1] - c0r;
  int64_t lo, hi;
  row_col_range<BLOCK>(A, B, r, b_sorted != 0, c_ncol, lo, hi);
  const bool multi = hi - lo > kRankCols;
  int64_t written = 0;
  for (int64_t s0 = lo; s0 < hi; s0 += kRankCols) {
    const int64_t s1 = hi < s0 + kRankCols ? hi : s0 + kRankCols;
    const int nw = (int)((s1 - s0 + 31) >> 5);
    const int32_t slot = saved_slot ? saved_slot[r] : -1;
    if (slot >= 0) {  // the symbolic kernel kept this row's bitmaps
      const uint32_t* src = saved + ((size_t)slot * saved_slices + (s0 - lo) / kRankCols) * (kRankCols / 32);
      for (int i = threadIdx.x; i < nw; i += BLOCK) bm[i] = src[i];
      __syncthreads();
    } else {
      for (int i = threadIdx.x; i < nw; i += BLOCK) bm[i] = 0u;
      __syncthreads();
      expand_row<BLOCK, false, VIn>(A, B, r, sg, multi, (int32_t)s0, (int32_t)s1,
                                    [&](int32_t key, VIn, VIn, int64_t) {
        const int64_t idx = (int64_t)key - s0;
        if (idx >= 0 && idx < kRankCols) atomicOr(&bm[idx >> 5], 1u << (idx & 31));
      });
      __syncthreads();
    }
    const int ng = (nw + 7) >> 3;
    long long run = 0;
    for (int g0 = 0; g0 < ng; g0 += BLOCK) {
      const int g = g0 + threadIdx.x;
      int cnt = 0;
      if (g < ng) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int w = g * 8 + k;
          wrank[w] = (uint16_t)cnt;
          cnt += w < nw ? __popc(bm[w]) : 0;
        }
      }
      long long tot;
      const long long ex = block_exclusive_sum<BLOCK, long long>((long long)cnt, sg.tmp, tot);
      if (g < ng) gbase[g] = (uint32_t)(run + ex);
      run += tot;
    }
    __syncthreads();
    const int64_t base = c0r + written;
    const int64_t room = nz - written;  // guards the writes if the counts disagree
    for (int w = threadIdx.x; w < nw; w += BLOCK) {
      uint32_t word = bm[w];
      int64_t pos = (int64_t)gbase[w >> 3] + wrank[w];
      while (word) {
        const int b = __ffs(word) - 1;
        word &= word - 1;
        if (pos < room) {
          ccol[base + pos] = (int32_t)(s0 + w * 32 + b);
          cval[base + pos] = AT(0);
        }
        ++pos;
      }
    }
    __syncthreads();  // the zeroed values are visible to the block's atomic adds
    expand_row<BLOCK, true, VIn>(A, B, r, sg, multi, (int32_t)s0, (int32_t)s1,
                                 [&](int32_t key, VIn av, VIn bv, int64_t) {
      const int64_t idx = (int64_t)key - s0;
      if (idx < 0 || idx >= kRankCols) return;
      const int w = (int)(idx >> 5);
      const int64_t pos = (int64_t)gbase[w >> 3] + wrank[w] + __popc(bm[w] & ((1u << (idx & 31)) - 1u));
      if (pos < room) Acc<VIn>::atomic_add(&cval[base + pos], Acc<VIn>::mul(av, bv));
    });
    written += run;
    __syncthreads();
  }
  if (threadIdx.x == 0 && written != nz) dev_report(st, written > nz ? kDevRowOverflow : kDevRowUnderflow, 13, r);
}

// ---- the heaviest rows over several blocks ----------------------------------
// A dense row with kSplitProducts products or more is split across blocks
// (the heavy-row regime the reference enters when the largest row's products
// pass SMTACT_*_THRES, src/ams/ams_utils.c:1538-1550, there by using every
// socket's cores).  k_dense_setup, one block per row, builds each column
// slice's bitmap (or takes the one the symbolic kernel kept), writes C's
// columns and zeroes its values as k_numc_dense does, and records for the
// parts: the bitmaps, the entries of C before each slice, the row's product
// prefix over its A entries and its part count.  k_dense_acc, a grid of
// persistent blocks, then takes parts (row, q) in ticket order, heaviest row
// first: part q of K takes the row's A entries whose products start in
// [q P / K, (q + 1) P / K), and for each slice loads the bitmap, ranks its
// words and adds its products into C by global atomics.  Because parts are
// taken row by row, only a few rows are being added into at any time, so
// their value ranges stay in L2, where the atomics resolve; a single block
// per row (k_numc_dense) keeps hundreds of rows of megabytes each open at
// once, and their atomics miss L2.
constexpr int kSplitLog2 = 17;
constexpr int64_t kSplitProducts = int64_t(1) << kSplitLog2;
constexpr int64_t kPartProducts = int64_t(1) << 17;

struct HeavyPlan {
  const int32_t* rows;      // the split rows, heaviest first
  int64_t n;                // their count
  int max_slices;           // column slices a row can span: ceil(columns / kRankCols)
  uint32_t* bits;           // n * max_slices bitmaps of kRankCols bits
  int64_t* slice_base;      // n * max_slices: entries of the row's C before each slice
  int64_t* lo;              // n: the row's first column
  int64_t* hi;              // n: one past the row's last column
  int32_t* nslices;         // n: slices the row spans
  int64_t* products;        // n: the row's products
  int64_t* nparts;          // n: parts of each row
  int64_t* parts;           // n + 1: the first part of each row (the scan of nparts), then the total
  int64_t* apre;            // per A entry of a split row (at its position in A): products of the
                            // row's earlier entries
  unsigned long long* ticket;
};

// Word ranks of a slice bitmap in shared memory: for each word the set bits
// of the words before it in its group of 8 (wrank) and the set bits before
// the group (gbase); returns the slice's set bits.
template <int BLOCK>
__device__ __forceinline__ long long slice_ranks(const uint32_t* __restrict__ bm, int nw, uint32_t* __restrict__ gbase,
                                                 uint16_t* __restrict__ wrank, long long* tmp) {
  const int ng = (nw + 7) >> 3;
  long long run = 0;
  for (int g0 = 0; g0 < ng; g0 += BLOCK) {
    const int g = g0 + threadIdx.x;
    int cnt = 0;
    if (g < ng) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int w = g * 8 + k;
        wrank[w] = (uint16_t)cnt;
        cnt += w < nw ? __popc(bm[w]) : 0;
      }
    }
    long long tot;
    const long long ex = block_exclusive_sum<BLOCK, long long>((long long)cnt, tmp, tot);
    if (g < ng) gbase[g] = (uint32_t)(run + ex);
    run += tot;
  }
  __syncthreads();
  return run;
}

// Exclusive scan of n counts into out[0..n], out[n] the total, by one block
// (the split rows are at most a few thousand).
__global__ void k_scan_one_block(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ out) {
  __shared__ long long tmp[33];
  long long run = 0;
  for (int64_t i0 = 0; i0 < n; i0 += 1024) {
    const int64_t i = i0 + threadIdx.x;
    const long long v = i < n ? in[i] : 0;
    long long tot;
    const long long ex = block_exclusive_sum<1024, long long>(v, tmp, tot);
    if (i < n) out[i] = run + ex;
    run += tot;
  }
  if (threadIdx.x == 0) out[n] = run;
}

template <int BLOCK, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_dense_setup(HeavyPlan hp, Csr A, Csr B, int64_t c_ncol, int32_t b_sorted, const int64_t* __restrict__ crp,
              int32_t* __restrict__ ccol, typename Acc<VIn>::T* __restrict__ cval, const uint32_t* __restrict__ saved,
              const int32_t* __restrict__ saved_slot, int saved_slices, const uint32_t* __restrict__ sym_bits,
              const int32_t* __restrict__ sym_slot, DevStatus* st) {
  using AT = typename Acc<VIn>::T;
  constexpr int NWORD = kRankCols / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem);
  uint32_t* gbase = bm + NWORD;
  uint16_t* wrank = reinterpret_cast<uint16_t*>(gbase + NWORD / 8);
  Stage<VIn>& sg = *reinterpret_cast<Stage<VIn>*>(reinterpret_cast<uint8_t*>(wrank + NWORD));
  const int64_t i = blockIdx.x;
  const int64_t r = hp.rows[i];
  const int64_t c0r = crp[r], nz = crp[r + 1] - c0r;
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  // the row's product prefix over its A entries, and its part count
  long long run = 0;
  for (int64_t a0 = as; a0 < ae; a0 += BLOCK) {
    long long len = 0;
    if (a0 + threadIdx.x < ae) {
      const int32_t k = A.col[a0 + threadIdx.x];
      len = B.rp[k + 1] - B.rp[k];
    }
    long long tot;
    const long long ex = block_exclusive_sum<BLOCK, long long>(len, sg.tmp, tot);
    if (a0 + threadIdx.x < ae) hp.apre[a0 + threadIdx.x] = run + ex;
    run += tot;
  }
  int64_t lo, hi;
  row_col_range<BLOCK>(A, B, r, b_sorted != 0, c_ncol, lo, hi);
  const int ns = hi > lo ? (int)((hi - lo + kRankCols - 1) / kRankCols) : 0;
  if (threadIdx.x == 0) {
    hp.products[i] = run;
    hp.nparts[i] = ns > 0 ? (run + kPartProducts - 1) / kPartProducts : 0;
    hp.lo[i] = lo;
    hp.hi[i] = hi;
    hp.nslices[i] = ns;
    if (ns > hp.max_slices) dev_report(st, kDevCapacity, 14, r);
  }
  const bool multi = ns > 1;
  int64_t written = 0;
  for (int sl = 0; sl < ns && sl < hp.max_slices; ++sl) {
    const int64_t s0 = lo + (int64_t)sl * kRankCols;
    const int64_t s1 = hi < s0 + kRankCols ? hi : s0 + kRankCols;
    const int nw = (int)((s1 - s0 + 31) >> 5);
    const int32_t slot = saved_slot ? saved_slot[r] : -1;
    const int32_t hslot = sym_slot ? sym_slot[r] : -1;  // the symbolic phase's split bitmaps
    if (hslot >= 0) {
      const uint32_t* src = sym_bits + ((size_t)hslot * hp.max_slices + sl) * NWORD;
      for (int w = threadIdx.x; w < nw; w += BLOCK) bm[w] = src[w];
      __syncthreads();
    } else if (slot >= 0) {
      const uint32_t* src = saved + ((size_t)slot * saved_slices + sl) * NWORD;
      for (int w = threadIdx.x; w < nw; w += BLOCK) bm[w] = src[w];
      __syncthreads();
    } else {
      for (int w = threadIdx.x; w < nw; w += BLOCK) bm[w] = 0u;
      __syncthreads();
      expand_row<BLOCK, false, VIn>(A, B, r, sg, multi, (int32_t)s0, (int32_t)s1, [&](int32_t key, VIn, VIn, int64_t) {
        const int64_t idx = (int64_t)key - s0;
        if (idx >= 0 && idx < kRankCols) atomicOr(&bm[idx >> 5], 1u << (idx & 31));
      });
      __syncthreads();
    }
    uint32_t* dst = hp.bits + ((size_t)i * hp.max_slices + sl) * NWORD;
    for (int w = threadIdx.x; w < nw; w += BLOCK) dst[w] = bm[w];
    if (threadIdx.x == 0) hp.slice_base[(size_t)i * hp.max_slices + sl] = written;
    const long long cnt = slice_ranks<BLOCK>(bm, nw, gbase, wrank, sg.tmp);
    const int64_t base = c0r + written;
    const int64_t room = nz - written;
    for (int w = threadIdx.x; w < nw; w += BLOCK) {
      uint32_t word = bm[w];
      int64_t pos = (int64_t)gbase[w >> 3] + wrank[w];
      while (word) {
        const int b = __ffs(word) - 1;
        word &= word - 1;
        if (pos < room) {
          ccol[base + pos] = (int32_t)(s0 + w * 32 + b);
          cval[base + pos] = AT(0);
        }
        ++pos;
      }
    }
    written += cnt;
    __syncthreads();
  }
  if (threadIdx.x == 0 && written != nz) dev_report(st, written > nz ? kDevRowOverflow : kDevRowUnderflow, 14, r);
}

template <int BLOCK, typename VIn>
__global__ void __launch_bounds__(BLOCK)
k_dense_acc(HeavyPlan hp, Csr A, Csr B, const int64_t* __restrict__ crp, typename Acc<VIn>::T* __restrict__ cval,
            DevStatus* st) {
  constexpr int NWORD = kRankCols / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem);
  uint32_t* gbase = bm + NWORD;
  uint16_t* wrank = reinterpret_cast<uint16_t*>(gbase + NWORD / 8);
  Stage<VIn>& sg = *reinterpret_cast<Stage<VIn>*>(reinterpret_cast<uint8_t*>(wrank + NWORD));
  __shared__ long long s_t, s_i;
  const int64_t total = hp.parts[hp.n];
  for (;;) {
    if (threadIdx.x == 0) {
      const long long t = (long long)atomicAdd(hp.ticket, 1ull);
      int64_t lo = 0, hi = hp.n;  // the row i with parts[i] <= t < parts[i + 1]
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (hp.parts[mid] <= t) lo = mid; else hi = mid;
      }
      s_t = t;
      s_i = lo;
    }
    __syncthreads();
    const int64_t t = s_t, i = s_i;
    __syncthreads();
    if (t >= total) break;
    const int64_t r = hp.rows[i];
    const int64_t K = hp.parts[i + 1] - hp.parts[i], q = t - hp.parts[i];
    const int64_t P = hp.products[i];
    const int64_t as = A.rp[r], ae = A.rp[r + 1];
    // A entries whose products start in [q P / K, (q + 1) P / K)
    auto first_at = [&](int64_t target) -> int64_t {  // first entry whose prefix is >= target
      int64_t l = as, h = ae;
      while (l < h) {
        const int64_t mid = (l + h) >> 1;
        if (hp.apre[mid] < target) l = mid + 1; else h = mid;
      }
      return l;
    };
    const int64_t a0 = q == 0 ? as : first_at(P * q / K);
    const int64_t a1 = q + 1 == K ? ae : first_at(P * (q + 1) / K);
    const int ns = hp.nslices[i];
    const int64_t lo = hp.lo[i], hi = hp.hi[i];
    const int64_t c0r = crp[r];
    for (int sl = 0; sl < ns && a1 > a0; ++sl) {
      const int64_t s0 = lo + (int64_t)sl * kRankCols;
      const int64_t s1 = hi < s0 + kRankCols ? hi : s0 + kRankCols;
      const int nw = (int)((s1 - s0 + 31) >> 5);
      const uint32_t* src = hp.bits + ((size_t)i * hp.max_slices + sl) * NWORD;
      const int64_t sb = hp.slice_base[(size_t)i * hp.max_slices + sl];
      for (int w = threadIdx.x; w < nw; w += BLOCK) bm[w] = src[w];
      __syncthreads();
      slice_ranks<BLOCK>(bm, nw, gbase, wrank, sg.tmp);
      const int64_t base = c0r + sb;
      expand_entries<BLOCK, true, VIn>(A, B, a0, a1, sg, ns > 1, (int32_t)s0, (int32_t)s1,
                                       [&](int32_t key, VIn av, VIn bv, int64_t) {
        const int64_t idx = (int64_t)key - s0;
        if (idx < 0 || idx >= s1 - s0) return;
        const int w = (int)(idx >> 5);
        const uint32_t m = bm[w];
        if (!((m >> (idx & 31)) & 1u)) return;  // cannot happen for a consistent bitmap
        const int64_t pos = (int64_t)gbase[w >> 3] + wrank[w] + __popc(m & ((1u << (idx & 31)) - 1u));
        Acc<VIn>::atomic_add(&cval[base + pos], Acc<VIn>::mul(av, bv));
      });
      __syncthreads();
    }
  }
}

// ---- symbolic bitmaps of the heaviest rows over several blocks ---------------
// The same split for the symbolic phase: the dense symbolic rows of at least
// kSplitProducts products are moved to their own list (k_split_dense_rows),
// one block per row plans the parts and clears the row's slice bitmaps
// (k_heavy_plan), persistent blocks take the parts in ticket order, build
// the part's bitmap of each slice in shared memory and OR its nonzero words
// into the row's bitmap in global memory (k_heavy_bits), and one block per
// row counts the bits (k_heavy_count: the row's distinct columns, and the
// entries before each slice).  The bitmaps stay for the numeric phase, whose
// setup copies them instead of expanding the row's products again.
__global__ void k_split_dense_rows(const int32_t* __restrict__ rows, int64_t n, const int64_t* __restrict__ row_flp,
                                   int64_t cap, int32_t* __restrict__ heavy, int32_t* __restrict__ light,
                                   unsigned long long* __restrict__ counts, int32_t* __restrict__ hslot) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = rows[i];
    bool h = row_flp[r] >= kSplitProducts;
    if (h) {
      const unsigned long long j = atomicAdd(&counts[0], 1ull);
      if ((int64_t)j < cap) {
        heavy[j] = r;
        hslot[r] = (int32_t)j;
      } else {
        h = false;
      }
    }
    if (!h) light[atomicAdd(&counts[1], 1ull)] = r;
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_heavy_plan(HeavyPlan hp, Csr A, Csr B, int64_t c_ncol, int32_t b_sorted, DevStatus* st) {
  __shared__ long long tmp[33];
  const int64_t i = blockIdx.x;
  const int64_t r = hp.rows[i];
  const int64_t as = A.rp[r], ae = A.rp[r + 1];
  long long run = 0;
  for (int64_t a0 = as; a0 < ae; a0 += BLOCK) {
    long long len = 0;
    if (a0 + threadIdx.x < ae) {
      const int32_t k = A.col[a0 + threadIdx.x];
      len = B.rp[k + 1] - B.rp[k];
    }
    long long tot;
    const long long ex = block_exclusive_sum<BLOCK, long long>(len, tmp, tot);
    if (a0 + threadIdx.x < ae) hp.apre[a0 + threadIdx.x] = run + ex;
    run += tot;
  }
  int64_t lo, hi;
  row_col_range<BLOCK>(A, B, r, b_sorted != 0, c_ncol, lo, hi);
  const int ns = hi > lo ? (int)((hi - lo + kRankCols - 1) / kRankCols) : 0;
  if (threadIdx.x == 0) {
    hp.products[i] = run;
    hp.nparts[i] = ns > 0 ? (run + kPartProducts - 1) / kPartProducts : 0;
    hp.lo[i] = lo;
    hp.hi[i] = hi;
    hp.nslices[i] = ns;
    if (ns > hp.max_slices) dev_report(st, kDevCapacity, 15, r);
  }
  uint32_t* bits = hp.bits + (size_t)i * hp.max_slices * (kRankCols / 32);
  const int64_t words = (int64_t)(ns < hp.max_slices ? ns : hp.max_slices) * (kRankCols / 32);
  for (int64_t w = threadIdx.x; w < words; w += BLOCK) bits[w] = 0u;
}
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_heavy_bits(HeavyPlan hp, Csr A, Csr B, DevStatus* st) {
  constexpr int NWORD = kRankCols / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem);
  Stage<double>& sg = *reinterpret_cast<Stage<double>*>(smem + NWORD * sizeof(uint32_t));
  __shared__ long long s_t, s_i;
  const int64_t total = hp.parts[hp.n];
  for (;;) {
    if (threadIdx.x == 0) {
      const long long t = (long long)atomicAdd(hp.ticket, 1ull);
      int64_t lo = 0, hi = hp.n;
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (hp.parts[mid] <= t) lo = mid; else hi = mid;
      }
      s_t = t;
      s_i = lo;
    }
    __syncthreads();
    const int64_t t = s_t, i = s_i;
    __syncthreads();
    if (t >= total) break;
    const int64_t r = hp.rows[i];
    const int64_t K = hp.parts[i + 1] - hp.parts[i], q = t - hp.parts[i];
    const int64_t P = hp.products[i];
    const int64_t as = A.rp[r], ae = A.rp[r + 1];
    auto first_at = [&](int64_t target) -> int64_t {
      int64_t l = as, h = ae;
      while (l < h) {
        const int64_t mid = (l + h) >> 1;
        if (hp.apre[mid] < target) l = mid + 1; else h = mid;
      }
      return l;
    };
    const int64_t a0 = q == 0 ? as : first_at(P * q / K);
    const int64_t a1 = q + 1 == K ? ae : first_at(P * (q + 1) / K);
    const int ns = hp.nslices[i] < hp.max_slices ? hp.nslices[i] : hp.max_slices;
    const int64_t lo = hp.lo[i], hi = hp.hi[i];
    for (int sl = 0; sl < ns && a1 > a0; ++sl) {
      const int64_t s0 = lo + (int64_t)sl * kRankCols;
      const int64_t s1 = hi < s0 + kRankCols ? hi : s0 + kRankCols;
      const int nw = (int)((s1 - s0 + 31) >> 5);
      for (int w = threadIdx.x; w < nw; w += BLOCK) bm[w] = 0u;
      __syncthreads();
      expand_entries<BLOCK, false, double>(A, B, a0, a1, sg, ns > 1, (int32_t)s0, (int32_t)s1,
                                           [&](int32_t key, double, double, int64_t) {
        const int64_t idx = (int64_t)key - s0;
        if (idx >= 0 && idx < s1 - s0) atomicOr(&bm[idx >> 5], 1u << (idx & 31));
      });
      __syncthreads();
      uint32_t* g = hp.bits + ((size_t)i * hp.max_slices + sl) * NWORD;
      for (int w = threadIdx.x; w < nw; w += BLOCK) {
        const uint32_t v = bm[w];
        if (v) atomicOr(&g[w], v);
      }
      __syncthreads();
    }
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_heavy_count(HeavyPlan hp, int64_t* __restrict__ row_nz) {
  __shared__ long long tmp[33];
  const int64_t i = blockIdx.x;
  const int ns = hp.nslices[i] < hp.max_slices ? hp.nslices[i] : hp.max_slices;
  const int64_t lo = hp.lo[i], hi = hp.hi[i];
  long long run = 0;
  for (int sl = 0; sl < ns; ++sl) {
    const int64_t s0 = lo + (int64_t)sl * kRankCols;
    const int64_t s1 = hi < s0 + kRankCols ? hi : s0 + kRankCols;
    const int nw = (int)((s1 - s0 + 31) >> 5);
    const uint32_t* g = hp.bits + ((size_t)i * hp.max_slices + sl) * (kRankCols / 32);
    long long c = 0;
    for (int w = threadIdx.x; w < nw; w += BLOCK) c += __popc(g[w]);
    c = block_sum<BLOCK, long long>(c, tmp);
    if (threadIdx.x == 0) hp.slice_base[(size_t)i * hp.max_slices + sl] = run;
    run += c;
  }
  if (threadIdx.x == 0) row_nz[hp.rows[i]] = run;
}
}  // namespace cas
