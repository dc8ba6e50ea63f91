// B = Aᵀ on the device (declared in include/casgemm.h).  Part of the
// cas_api.cu translation unit.
//
// The reference makes B on the host and reads it from disk: trpl_transpose
// (src/mm/mm_utils.c:742-754) swaps each triple's row and column and sorts
// the triples by (row, column), txt_transpose (:851-862) writes them as
// <dataset>.trs.mtx, and every driver reads that file as its second input.
// Here B comes from A on the device, as a stable counting sort of A's
// entries by column, so each row of B lists A's rows in increasing order and
// duplicate (row, column) entries keep A's order: entry for entry the result
// of the host's counting-sort transpose (cas_csr_transpose_host).
//
//   k_tr_count     entries per column (lanes of a warp that hit the same
//                  column add once: hot columns of a skewed matrix take one
//                  atomic per warp instead of one per entry)
//   scan           B's row pointers
//   k_tr_scatter   each entry's position in A to the next free slot of its
//                  column (warp-aggregated in the same way)
//   k_tr_sort_warp / k_tr_sort_block
//                  each row of B sorted by those positions: a warp bitonic
//                  sort for rows of at most 32 entries, a block's stable LSD
//                  radix sort (8-bit digits, only the bits the row spans)
//                  for longer ones
//   k_tr_gather    B's column (A's row, found by binary search in A's row
//                  pointers) and value of each entry
namespace {

constexpr int kTrBlock = 256;

__global__ void k_tr_count(int64_t nnz, const int32_t* __restrict__ col, unsigned long long* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nnz; base += stride) {
    const int64_t e = base + lane;
    const int c = e < nnz ? col[e] : -1;
    const unsigned peers = __match_any_sync(cas::kFull, c);
    if (c >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cnt[c], (unsigned long long)__popc(peers));
  }
}

__global__ void k_tr_scatter(int64_t nnz, const int32_t* __restrict__ col, unsigned long long* __restrict__ cur,
                             unsigned long long* __restrict__ key) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nnz; base += stride) {
    const int64_t e = base + lane;
    const int c = e < nnz ? col[e] : -1;
    const unsigned peers = __match_any_sync(cas::kFull, c);
    if (c >= 0) {
      const int leader = __ffs(peers) - 1;
      unsigned long long b = 0;
      if (lane == leader) b = atomicAdd(&cur[c], (unsigned long long)__popc(peers));
      b = __shfl_sync(peers, b, leader);
      key[b + __popc(peers & cas::lanemask_lt())] = (unsigned long long)e;
    }
  }
}

// Rows of at most 32 entries: a warp per row, one entry per lane, bitonic
// sort in registers.  Longer rows are listed for k_tr_sort_block.
__global__ void k_tr_sort_warp(int64_t n, const int64_t* __restrict__ rp, unsigned long long* __restrict__ key,
                               int32_t* __restrict__ big, unsigned int* __restrict__ nbig) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += warps) {
    const int64_t s = rp[j], len = rp[j + 1] - s;
    if (len <= 1) continue;
    if (len > 32) {
      if (lane == 0) big[atomicAdd(nbig, 1u)] = (int32_t)j;
      continue;
    }
    unsigned long long v = lane < len ? key[s + lane] : ~0ull;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int m = k >> 1; m > 0; m >>= 1) {
        const unsigned long long o = __shfl_xor_sync(cas::kFull, v, m);
        const bool up = (lane & k) == 0;
        const bool lower = (lane & m) == 0;
        v = (lower == up) ? (v < o ? v : o) : (v < o ? o : v);
      }
    }
    if (lane < len) key[s + lane] = v;
  }
}

// Longer rows: a block per row, a stable LSD radix sort of (position - the
// row's smallest position) by 8-bit digits over only the bits the row spans.
// Each pass runs over the row in tiles of kTrBlock entries in order; within a
// tile an entry's place is its digit's running offset, plus the counts of
// that digit in earlier warps of the tile, plus its rank among the lanes of
// its warp with the same digit, so equal digits keep their order.  The passes
// alternate between `key` and `aux` (the same offsets); an odd number of
// passes ends with a copy back.
__global__ void __launch_bounds__(kTrBlock) k_tr_sort_block(const int64_t* __restrict__ rp,
                                                            const int32_t* __restrict__ big,
                                                            unsigned long long* __restrict__ key,
                                                            unsigned long long* __restrict__ aux) {
  constexpr int NW = kTrBlock / 32;
  __shared__ unsigned int hist[256];
  __shared__ unsigned int run[256];
  __shared__ unsigned int wcnt[NW][257];
  __shared__ unsigned long long s_min, s_max;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t j = big[blockIdx.x];
  const int64_t s = rp[j], len = rp[j + 1] - s;
  if (threadIdx.x == 0) {
    s_min = ~0ull;
    s_max = 0ull;
  }
  __syncthreads();
  unsigned long long mn = ~0ull, mx = 0ull;
  for (int64_t i = threadIdx.x; i < len; i += kTrBlock) {
    const unsigned long long v = key[s + i];
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
  atomicMin(&s_min, mn);
  atomicMax(&s_max, mx);
  __syncthreads();
  const unsigned long long kmin = s_min, span = s_max - s_min;
  const int bits = span ? 64 - __clzll((long long)span) : 0;
  const int passes = (bits + 7) / 8;
  unsigned long long* src = key;
  unsigned long long* dst = aux;
  for (int pass = 0; pass < passes; ++pass) {
    const int sh = pass * 8;
    for (int d = threadIdx.x; d < 256; d += kTrBlock) hist[d] = 0u;
    __syncthreads();
    for (int64_t i = threadIdx.x; i < len; i += kTrBlock) atomicAdd(&hist[((src[s + i] - kmin) >> sh) & 0xFF], 1u);
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the 256 digit counts: 8 per lane
      unsigned int c[8], t = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        c[q] = hist[lane * 8 + q];
        t += c[q];
      }
      unsigned int ex = cas::warp_inclusive_sum(t) - t;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        run[lane * 8 + q] = ex;
        ex += c[q];
      }
    }
    for (int i = threadIdx.x; i < NW * 257; i += kTrBlock) (&wcnt[0][0])[i] = 0u;
    __syncthreads();
    for (int64_t t0 = 0; t0 < len; t0 += kTrBlock) {
      const int64_t i = t0 + threadIdx.x;
      const bool ok = i < len;
      const unsigned long long v = ok ? src[s + i] : 0ull;
      const int d = ok ? (int)(((v - kmin) >> sh) & 0xFF) : 256;
      const unsigned peers = __match_any_sync(cas::kFull, d);
      const int rank = __popc(peers & cas::lanemask_lt());
      if (lane == __ffs(peers) - 1) wcnt[warp][d] = (unsigned int)__popc(peers);
      __syncthreads();
      if (threadIdx.x < 256) {  // per digit: offsets of the warps' runs, in warp order
        const int dd = threadIdx.x;
        unsigned int r = run[dd];
        for (int w = 0; w < NW; ++w) {
          const unsigned int c = wcnt[w][dd];
          wcnt[w][dd] = r;
          r += c;
        }
        run[dd] = r;
      }
      __syncthreads();
      if (ok) dst[s + wcnt[warp][d] + rank] = v;
      __syncthreads();
      for (int q = threadIdx.x; q < NW * 257; q += kTrBlock) (&wcnt[0][0])[q] = 0u;
      __syncthreads();
    }
    unsigned long long* t = src;
    src = dst;
    dst = t;
  }
  if (passes & 1)
    for (int64_t i = threadIdx.x; i < len; i += kTrBlock) key[s + i] = aux[s + i];
}

template <typename V>
__global__ void k_tr_gather(int64_t nnz, int64_t m, const int64_t* __restrict__ arp, const V* __restrict__ aval,
                            const unsigned long long* __restrict__ key, int32_t* __restrict__ bcol,
                            V* __restrict__ bval) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = (int64_t)key[p];
    int64_t lo = 0, hi = m;  // the row i with arp[i] <= e < arp[i + 1]
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (arp[mid] <= e) lo = mid; else hi = mid;
    }
    bcol[p] = (int32_t)lo;
    bval[p] = aval[e];
  }
}

cas_status transpose_device(cas_ctx* ctx, const DevMat& A, int vt, cas_csr* B, bool to_host, double& d2h) {
  const int64_t m = A.csr.nrow, n = A.csr.ncol, nnz = A.nnz;
  const size_t vbytes = vt == CAS_VAL_F64 ? 8 : 4;
  int64_t *brp = nullptr, *cnt = nullptr, *partial = nullptr;
  int32_t *bcol = nullptr, *big = nullptr;
  void* bval = nullptr;
  unsigned long long *key = nullptr, *aux = nullptr;
  unsigned int* nbig = reinterpret_cast<unsigned int*>(ctx->d_counts + kSlotOvf);
  std::vector<void*> tmp;
  auto release = [&]() {
    for (void* p : tmp) cudaFreeAsync(p, ctx->stream);
  };
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(dev_alloc(ctx, (void**)&brp, sizeof(int64_t) * (size_t)(n + 1)));
    CAS_TRY(dev_alloc(ctx, (void**)&bcol, sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1)));
    CAS_TRY(dev_alloc(ctx, &bval, vbytes * (size_t)(nnz > 0 ? nnz : 1)));
    CAS_TRY(dev_alloc(ctx, (void**)&cnt, sizeof(int64_t) * (size_t)(n + 1)));
    tmp.push_back(cnt);
    CAS_TRY(dev_alloc(ctx, (void**)&partial, sizeof(int64_t) * (size_t)((n + 1 + cas::kScanTile - 1) / cas::kScanTile + 1)));
    tmp.push_back(partial);
    CAS_TRY(dev_alloc(ctx, (void**)&key, sizeof(unsigned long long) * (size_t)(nnz > 0 ? nnz : 1)));
    tmp.push_back(key);
    CAS_TRY(dev_alloc(ctx, (void**)&aux, sizeof(unsigned long long) * (size_t)(nnz > 0 ? nnz : 1)));
    tmp.push_back(aux);
    CAS_TRY(dev_alloc(ctx, (void**)&big, sizeof(int32_t) * (size_t)(n > 0 ? n : 1)));
    tmp.push_back(big);
    CAS_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t) * (size_t)(n + 1), ctx->stream));
    CAS_CUDA(ctx, cudaMemsetAsync(nbig, 0, sizeof(unsigned int), ctx->stream));
    const int g = grid_for(nnz, kTrBlock, ctx->sm_count * 8);
    if (nnz > 0) {
      k_tr_count<<<g, kTrBlock, 0, ctx->stream>>>(nnz, A.csr.col, reinterpret_cast<unsigned long long*>(cnt));
      CAS_TRY(check_launch(ctx, "k_tr_count"));
    }
    CAS_TRY(launch_scan(ctx, brp, cnt, n + 1, partial, nullptr));
    if (nnz > 0) {
      CAS_CUDA(ctx, cudaMemcpyAsync(cnt, brp, sizeof(int64_t) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
      k_tr_scatter<<<g, kTrBlock, 0, ctx->stream>>>(nnz, A.csr.col, reinterpret_cast<unsigned long long*>(cnt), key);
      CAS_TRY(check_launch(ctx, "k_tr_scatter"));
      k_tr_sort_warp<<<grid_for(n * 32, kTrBlock, ctx->sm_count * 16), kTrBlock, 0, ctx->stream>>>(n, brp, key, big,
                                                                                                  nbig);
      CAS_TRY(check_launch(ctx, "k_tr_sort_warp"));
      unsigned int nb = 0;
      CAS_CUDA(ctx, cudaMemcpyAsync(&nb, nbig, sizeof(nb), cudaMemcpyDeviceToHost, ctx->stream));
      CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (nb > 0) {
        k_tr_sort_block<<<nb, kTrBlock, 0, ctx->stream>>>(brp, big, key, aux);
        CAS_TRY(check_launch(ctx, "k_tr_sort_block"));
      }
      if (vt == CAS_VAL_F64)
        k_tr_gather<double><<<g, kTrBlock, 0, ctx->stream>>>(nnz, m, A.csr.rp, static_cast<const double*>(A.csr.val),
                                                             key, bcol, static_cast<double*>(bval));
      else
        k_tr_gather<int32_t><<<g, kTrBlock, 0, ctx->stream>>>(nnz, m, A.csr.rp,
                                                              static_cast<const int32_t*>(A.csr.val), key, bcol,
                                                              static_cast<int32_t*>(bval));
      CAS_TRY(check_launch(ctx, "k_tr_gather"));
    }
    memset(B, 0, sizeof(*B));
    B->num_row = n;
    B->num_col = m;
    B->num_nnz = nnz;
    B->col_bytes = 4;
    B->val_type = vt;
    B->owned = 1;
    if (!to_host) {
      B->on_device = 1;
      B->row_ptrs = brp;
      B->cols = bcol;
      B->rats = bval;
      brp = nullptr;
      bcol = nullptr;
      bval = nullptr;
      return CAS_OK;
    }
    B->on_device = 0;
    B->row_ptrs = static_cast<int64_t*>(malloc(sizeof(int64_t) * (size_t)(n + 1)));
    B->cols = malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    B->rats = malloc(vbytes * (size_t)(nnz > 0 ? nnz : 1));
    if (!B->row_ptrs || !B->cols || !B->rats) {
      free(B->row_ptrs);
      free(B->cols);
      free(B->rats);
      memset(B, 0, sizeof(*B));
      return set_err(ctx, CAS_ERR_OOM, "host allocation of the transpose failed");
    }
    CAS_CUDA(ctx, cudaMemcpyAsync(B->row_ptrs, brp, sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(B->cols, bcol, sizeof(int32_t) * (size_t)nnz, cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(B->rats, bval, vbytes * (size_t)nnz, cudaMemcpyDeviceToHost, ctx->stream));
    d2h += sizeof(int64_t) * (double)(n + 1) + (4.0 + (double)vbytes) * (double)nnz;
    return CAS_OK;
  }();
  if (brp) tmp.push_back(brp);
  if (bcol) tmp.push_back(bcol);
  if (bval) tmp.push_back(bval);
  release();
  cudaStreamSynchronize(ctx->stream);
  return rc;
}

}  // namespace

extern "C" cas_status cas_csr_transpose(cas_ctx* ctx, const cas_csr* A, cas_csr* B) {
  if (!ctx || !B) return CAS_ERR_BAD_INPUT;
  CAS_TRY(basic_checks(ctx, A, "A"));
  CAS_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaGetLastError();
  const bool to_host = B->on_device == 0;
  DevMat dA;
  double h2d = 0, d2h = 0;
  cas_status rc = to_device(ctx, A, dA, h2d);
  if (rc == CAS_OK) {  // check the input's structure on the device, as cas_spgemm does
    CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts, 0, sizeof(unsigned long long) * kCountSlots, ctx->stream));
    cas::Csr a = dA.csr;
    if (a.nrow > 0) {
      cas::k_check_csr<<<grid_for(a.nrow * 32, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
          a, A->num_nnz, ctx->d_counts + kSlotCheck);
      rc = check_launch(ctx, "k_check_csr");
      if (rc == CAS_OK) {
        unsigned long long bad = 0;
        if (cudaMemcpyAsync(&bad, ctx->d_counts + kSlotCheck, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
          rc = set_err(ctx, CAS_ERR_CUDA, "structure check of A failed");
        else if (bad)
          rc = set_err(ctx, CAS_ERR_BAD_INPUT, "A's row pointers or columns are out of range");
      }
    }
  }
  if (rc == CAS_OK) rc = transpose_device(ctx, dA, A->val_type, B, to_host, d2h);
  free_owned(ctx, dA);
  cudaStreamSynchronize(ctx->stream);
  ctx->stats.h2d_bytes = h2d;
  ctx->stats.d2h_bytes = d2h;
  return rc;
}
