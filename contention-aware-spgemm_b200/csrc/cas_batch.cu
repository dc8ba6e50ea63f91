// Digests and batches of independent products (declared in include/casgemm.h).
// Part of the cas_api.cu translation unit: it drives the same pipeline
// (run_spgemm) and uses its error and allocation helpers.
//
// CAS_BATCH_WAVES packs every job into one block-diagonal product
//   diag(A_1, ..., A_n) * diag(B_1, ..., B_n) = diag(C_1, ..., C_n):
// the jobs' CSRs are copied into one device CSR pair, A's columns shifted by
// the rows of the B blocks before them and B's columns by the columns of the
// B blocks before them.  A row of the packed product is a row of one job, so
// every bin kernel of a wave serves rows of many jobs in one launch, and the
// rows of a large job can split across waves.  Waves are cut so that the
// bound 12 bytes * min(products, columns of the job) per row stays within
// the budget.  A digest kernel folds each wave's rows into per-job digests,
// subtracting each row's column shift, and the wave's C is released.
// CAS_BATCH_PER_CALL runs one cas_spgemm per job with the same kernels, and
// CAS_BATCH_CONCURRENT runs them so on several host threads and streams.

namespace cas {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t val_bits(double v) { return (uint64_t)__double_as_longlong(v); }
__device__ __forceinline__ uint64_t val_bits(long long v) { return (uint64_t)v; }

// One warp per row of a product's rows [0, m) (global row g0 + r of the
// batch): the row digest, folded into its job's digest.  job_of == nullptr
// means a single job 0 with no shifts, whose rows [0, m) are its rows
// [g0, g0 + m) (a row chunk of a larger product).
template <typename OT>
__global__ void __launch_bounds__(256)
k_row_digest(int64_t m, int64_t g0, const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
             const OT* __restrict__ val, const int32_t* __restrict__ job_of, const int64_t* __restrict__ row_base,
             const int64_t* __restrict__ col_base, unsigned long long* __restrict__ job_digest,
             unsigned long long* __restrict__ job_nnz, uint64_t* __restrict__ row_digest) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t g = g0 + r;
    const int j = job_of ? job_of[g] : 0;
    const int64_t rloc = job_of ? g - row_base[j] : g;
    const uint64_t cb = job_of ? (uint64_t)col_base[j] : 0ull;
    const int64_t s = rp[r], e = rp[r + 1];
    uint64_t h = 0;
    for (int64_t k = s + lane; k < e; k += 32) {
      const uint64_t c = (uint64_t)(uint32_t)col[k] - cb;
      h += mix64(c * 0x9E3779B97F4A7C15ull + (uint64_t)(k - s)) ^ mix64(val_bits(val[k]) + 0x632BE59BD9B4E019ull);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) h += __shfl_xor_sync(kFull, h, d);
    if (lane == 0) {
      if (row_digest) row_digest[g] = h;
      atomicAdd(job_digest + j, (unsigned long long)mix64(h + (uint64_t)rloc));
      atomicAdd(job_nnz + j, (unsigned long long)(e - s));
    }
  }
}

// job_of[g] for the packed rows: the job whose [base[j], base[j+1]) holds g.
__global__ void k_fill_job_of(int64_t rows, const int64_t* __restrict__ base, int njobs, int32_t* __restrict__ job_of) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < rows; g += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = njobs;  // last j with base[j] <= g
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (base[mid] <= g) lo = mid; else hi = mid;
    }
    job_of[g] = lo;
  }
}

// Shifts the packed row pointers by the entries of the jobs before each row.
__global__ void k_shift_rows(int64_t rows, int64_t* __restrict__ rp, const int32_t* __restrict__ job_of,
                             const int64_t* __restrict__ nnz_base) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < rows; g += (int64_t)gridDim.x * blockDim.x)
    rp[g] += nnz_base[job_of[g]];
}

// Shifts the packed columns by their job's column base, after checking each
// against the job's own column count (flag[0] set on a bad index).  Each
// block takes a tile of kShiftTile entries and walks the job boundaries.
constexpr int kShiftTile = 4096;
__global__ void k_shift_cols(int64_t nnz, int32_t* __restrict__ col, const int64_t* __restrict__ nnz_base, int njobs,
                             const int64_t* __restrict__ col_base, const int64_t* __restrict__ ncol,
                             unsigned long long* __restrict__ flag) {
  for (int64_t t0 = (int64_t)blockIdx.x * kShiftTile; t0 < nnz; t0 += (int64_t)gridDim.x * kShiftTile) {
    int lo = 0, hi = njobs;  // job of the tile's first entry
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (nnz_base[mid] <= t0) lo = mid; else hi = mid;
    }
    const int64_t t1 = t0 + kShiftTile < nnz ? t0 + kShiftTile : nnz;
    for (int64_t e = t0 + threadIdx.x; e < t1; e += blockDim.x) {
      int j = lo;
      while (j + 1 < njobs && nnz_base[j + 1] <= e) ++j;
      const int32_t c = col[e];
      if (c < 0 || (int64_t)c >= ncol[j]) {
        atomicOr(flag, 1ull);
        continue;
      }
      col[e] = (int32_t)(c + col_base[j]);
    }
  }
}

// Row products of the packed A against the packed B, and the per-row output
// bound min(products, columns of the row's job).
__global__ void k_row_products(int64_t rows, const int64_t* __restrict__ arp, const int32_t* __restrict__ acol,
                               const int64_t* __restrict__ brp, const int32_t* __restrict__ job_of,
                               const int64_t* __restrict__ ncol, int64_t* __restrict__ flp,
                               int64_t* __restrict__ bound) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < rows; g += nw) {
    long long p = 0;
    for (int64_t k = arp[g] + lane; k < arp[g + 1]; k += 32) {
      const int32_t c = acol[k];
      p += brp[c + 1] - brp[c];
    }
    p = warp_sum(p);
    if (lane == 0) {
      flp[g] = p;
      const int64_t nc = ncol[job_of[g]];
      bound[g] = p < nc ? p : nc;
    }
  }
}

}  // namespace cas

namespace {

struct Packed {
  int64_t rows = 0, nnz = 0, ncol = 0;
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  void* val = nullptr;
  int32_t* job_of = nullptr;
  int64_t *d_row_base = nullptr, *d_nnz_base = nullptr, *d_col_base = nullptr, *d_ncol = nullptr;
  std::vector<int64_t> row_base, nnz_base, col_base, ncol_of;
};

cas_status packed_free(cas_ctx* ctx, Packed& p) {
  void* ps[] = {p.rp, p.col, p.val, p.job_of, p.d_row_base, p.d_nnz_base, p.d_col_base, p.d_ncol};
  for (void* q : ps)
    if (q) CAS_CUDA(ctx, cudaFreeAsync(q, ctx->stream));
  p = Packed();
  return CAS_OK;
}

cas_status upload_i64(cas_ctx* ctx, int64_t** d, const std::vector<int64_t>& h) {
  CAS_TRY(dev_alloc(ctx, (void**)d, sizeof(int64_t) * h.size()));
  CAS_CUDA(ctx, cudaMemcpyAsync(*d, h.data(), sizeof(int64_t) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
  return CAS_OK;
}

// Packs side `which` (0: A, 1: B) of every job into one device CSR.  The
// columns of A shift by the rows of the B blocks before it; those of B by
// the columns of the B blocks before it.
cas_status pack_side(cas_ctx* ctx, const cas_job* jobs, int64_t n, int which, size_t vbytes, Packed& P,
                     double& h2d) {
  using namespace cas;
  P.row_base.assign(n + 1, 0);
  P.nnz_base.assign(n + 1, 0);
  P.col_base.assign(n + 1, 0);
  P.ncol_of.assign(n, 0);
  for (int64_t j = 0; j < n; ++j) {
    const cas_csr& M = which == 0 ? jobs[j].A : jobs[j].B;
    P.row_base[j + 1] = P.row_base[j] + M.num_row;
    P.nnz_base[j + 1] = P.nnz_base[j] + M.num_nnz;
    P.col_base[j + 1] = P.col_base[j] + (which == 0 ? jobs[j].B.num_row : M.num_col);
    P.ncol_of[j] = M.num_col;
  }
  P.rows = P.row_base[n];
  P.nnz = P.nnz_base[n];
  P.ncol = P.col_base[n];
  if (P.rows > INT32_MAX || P.ncol > INT32_MAX)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "packed batch has %lld rows and %lld columns; at most 2^31-1 each",
                   (long long)P.rows, (long long)P.ncol);
  CAS_TRY(dev_alloc(ctx, (void**)&P.rp, sizeof(int64_t) * (P.rows + 1)));
  CAS_TRY(dev_alloc(ctx, (void**)&P.col, sizeof(int32_t) * P.nnz));
  CAS_TRY(dev_alloc(ctx, &P.val, vbytes * P.nnz));
  CAS_TRY(dev_alloc(ctx, (void**)&P.job_of, sizeof(int32_t) * (P.rows + 1)));
  CAS_TRY(upload_i64(ctx, &P.d_row_base, P.row_base));
  CAS_TRY(upload_i64(ctx, &P.d_nnz_base, P.nnz_base));
  CAS_TRY(upload_i64(ctx, &P.d_col_base, P.col_base));
  CAS_TRY(upload_i64(ctx, &P.d_ncol, P.ncol_of));
  for (int64_t j = 0; j < n; ++j) {
    const cas_csr& M = which == 0 ? jobs[j].A : jobs[j].B;
    const cudaMemcpyKind kind = M.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (M.num_row > 0)
      CAS_CUDA(ctx, cudaMemcpyAsync(P.rp + P.row_base[j], M.row_ptrs, sizeof(int64_t) * M.num_row, kind, ctx->stream));
    if (M.num_nnz > 0) {
      CAS_CUDA(ctx, cudaMemcpyAsync(P.col + P.nnz_base[j], M.cols, sizeof(int32_t) * M.num_nnz, kind, ctx->stream));
      CAS_CUDA(ctx, cudaMemcpyAsync(static_cast<char*>(P.val) + vbytes * P.nnz_base[j], M.rats, vbytes * M.num_nnz,
                                    kind, ctx->stream));
    }
    if (!M.on_device) h2d += sizeof(int64_t) * (double)M.num_row + (4.0 + vbytes) * (double)M.num_nnz;
  }
  CAS_CUDA(ctx, cudaMemcpyAsync(P.rp + P.rows, &P.nnz_base[n], sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
  const int g = grid_for(P.rows, 256, ctx->sm_count * 8);
  if (P.rows > 0) {
    k_fill_job_of<<<g, 256, 0, ctx->stream>>>(P.rows, P.d_row_base, (int)n, P.job_of);
    CAS_TRY(check_launch(ctx, "k_fill_job_of"));
    k_shift_rows<<<g, 256, 0, ctx->stream>>>(P.rows, P.rp, P.job_of, P.d_nnz_base);
    CAS_TRY(check_launch(ctx, "k_shift_rows"));
  }
  if (P.nnz > 0) {
    CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotCheck, 0, sizeof(unsigned long long), ctx->stream));
    k_shift_cols<<<grid_for(P.nnz, kShiftTile, ctx->sm_count * 8), 256, 0, ctx->stream>>>(
        P.nnz, P.col, P.d_nnz_base, (int)n, P.d_col_base, P.d_ncol, ctx->d_counts + kSlotCheck);
    CAS_TRY(check_launch(ctx, "k_shift_cols"));
    CAS_CUDA(ctx, cudaMemcpyAsync(ctx->h_counts + kSlotCheck, ctx->d_counts + kSlotCheck, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->h_counts[kSlotCheck])
      return set_err(ctx, CAS_ERR_BAD_INPUT, "a job of the batch has a column index outside its matrix");
  }
  return CAS_OK;
}

cas_status digest_launch(cas_ctx* ctx, const cas_csr& C, int64_t g0, const int32_t* job_of, const int64_t* row_base,
                         const int64_t* col_base, unsigned long long* job_digest, unsigned long long* job_nnz,
                         uint64_t* row_digest) {
  using namespace cas;
  if (C.num_row <= 0) return CAS_OK;
  const int g = grid_for(C.num_row * 32, 256, ctx->sm_count * 8);
  const int32_t* col = static_cast<const int32_t*>(C.cols);
  if (C.val_type == CAS_VAL_F64)
    k_row_digest<double><<<g, 256, 0, ctx->stream>>>(C.num_row, g0, C.row_ptrs, col, static_cast<const double*>(C.rats),
                                                     job_of, row_base, col_base, job_digest, job_nnz, row_digest);
  else
    k_row_digest<long long><<<g, 256, 0, ctx->stream>>>(C.num_row, g0, C.row_ptrs, col,
                                                        static_cast<const long long*>(C.rats), job_of, row_base,
                                                        col_base, job_digest, job_nnz, row_digest);
  return check_launch(ctx, "k_row_digest");
}

struct BatchOut {
  unsigned long long* digest = nullptr;  // device, one per job
  unsigned long long* nnz = nullptr;
  uint64_t* rows = nullptr;              // device per-row digests (packed rows), or nullptr
  int64_t nrows = 0;
};

cas_status batch_out_alloc(cas_ctx* ctx, int64_t n, int64_t nrows, bool rows, BatchOut& o) {
  CAS_TRY(dev_alloc(ctx, (void**)&o.digest, sizeof(unsigned long long) * n));
  CAS_TRY(dev_alloc(ctx, (void**)&o.nnz, sizeof(unsigned long long) * n));
  CAS_CUDA(ctx, cudaMemsetAsync(o.digest, 0, sizeof(unsigned long long) * n, ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(o.nnz, 0, sizeof(unsigned long long) * n, ctx->stream));
  o.nrows = nrows;
  if (rows) CAS_TRY(dev_alloc(ctx, (void**)&o.rows, sizeof(uint64_t) * (nrows > 0 ? nrows : 1)));
  return CAS_OK;
}

cas_status batch_out_free(cas_ctx* ctx, BatchOut& o) {
  void* ps[] = {o.digest, o.nnz, o.rows};
  for (void* q : ps)
    if (q) CAS_CUDA(ctx, cudaFreeAsync(q, ctx->stream));
  o = BatchOut();
  return CAS_OK;
}

cas_status batch_waves(cas_ctx* ctx, cas_accum accum, cas_job* jobs, int64_t n, double budget, size_t vbytes,
                       cas_batch_stats& st) {
  using namespace cas;
  Packed PA, PB;
  BatchOut out;
  int64_t *flp = nullptr, *bound = nullptr;
  bool want_rows = false;
  for (int64_t j = 0; j < n; ++j) want_rows |= jobs[j].row_digests != nullptr;
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(pack_side(ctx, jobs, n, 1, vbytes, PB, st.h2d_bytes));
    CAS_TRY(pack_side(ctx, jobs, n, 0, vbytes, PA, st.h2d_bytes));
    // A's packed columns index the packed B's rows
    PA.ncol = PB.rows;
    CAS_TRY(batch_out_alloc(ctx, n, PA.rows, want_rows, out));
    // per-row products and output bounds, planned into waves on the host
    CAS_TRY(dev_alloc(ctx, (void**)&flp, sizeof(int64_t) * (PA.rows + 1)));
    CAS_TRY(dev_alloc(ctx, (void**)&bound, sizeof(int64_t) * (PA.rows + 1)));
    if (PA.rows > 0) {
      k_row_products<<<grid_for(PA.rows * 32, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(
          PA.rows, PA.rp, PA.col, PB.rp, PA.job_of, PB.d_ncol, flp, bound);
      CAS_TRY(check_launch(ctx, "k_row_products"));
    }
    std::vector<int64_t> h_flp((size_t)PA.rows), h_bound((size_t)PA.rows);
    CAS_CUDA(ctx, cudaMemcpyAsync(h_flp.data(), flp, sizeof(int64_t) * PA.rows, cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(h_bound.data(), bound, sizeof(int64_t) * PA.rows, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t j = 0; j < n; ++j) {
      int64_t f = 0;
      for (int64_t g = PA.row_base[j]; g < PA.row_base[j + 1]; ++g) f += h_flp[(size_t)g];
      jobs[j].flop = f;
      st.flop += f;
    }
    // waves: contiguous packed rows whose output bound (12 bytes per entry,
    // plus 48 bytes of per-row scratch) fits the budget
    std::vector<int64_t> cut{0};
    double acc = 0;
    for (int64_t g = 0; g < PA.rows; ++g) {
      const double b = 12.0 * (double)h_bound[(size_t)g] + 48.0;
      if (acc + b > budget && g > cut.back()) {
        st.max_wave_bound = std::max(st.max_wave_bound, acc);
        cut.push_back(g);
        acc = 0;
      }
      acc += b;
    }
    st.max_wave_bound = std::max(st.max_wave_bound, acc);
    if (cut.back() != PA.rows) cut.push_back(PA.rows);
    CAS_CUDA(ctx, cudaFreeAsync(flp, ctx->stream));
    CAS_CUDA(ctx, cudaFreeAsync(bound, ctx->stream));
    flp = bound = nullptr;
    // the waves: row slices of the packed A against the whole packed B
    cas_csr b_view{};
    b_view.num_row = PB.rows;
    b_view.num_col = PB.ncol;
    b_view.num_nnz = PB.nnz;
    b_view.row_ptrs = PB.rp;
    b_view.cols = PB.col;
    b_view.rats = PB.val;
    b_view.col_bytes = 4;
    b_view.val_type = jobs[0].A.val_type;
    b_view.on_device = 1;
    for (size_t w = 0; w + 1 < cut.size(); ++w) {
      const int64_t g0 = cut[w], g1 = cut[w + 1];
      cas_csr a_view = b_view;
      a_view.num_row = g1 - g0;
      a_view.num_col = PA.ncol;
      a_view.num_nnz = PA.nnz;  // the row pointers index the whole packed arrays
      a_view.row_ptrs = PA.rp + g0;
      a_view.cols = PA.col;
      a_view.rats = PA.val;
      cas_csr C{};
      C.on_device = 1;
      CAS_TRY(run_spgemm(ctx, accum, &a_view, &b_view, &C, nullptr));
      st.nnz_c += C.num_nnz;
      cas_status ds = digest_launch(ctx, C, g0, PA.job_of, PA.d_row_base, PB.d_col_base, out.digest, out.nnz, out.rows);
      cas_csr_free(ctx, &C);
      CAS_TRY(ds);
      st.waves++;
    }
    // results
    std::vector<unsigned long long> hd((size_t)n), hn((size_t)n);
    CAS_CUDA(ctx, cudaMemcpyAsync(hd.data(), out.digest, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(hn.data(), out.nnz, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    for (int64_t j = 0; j < n; ++j)
      if (jobs[j].row_digests && jobs[j].A.num_row > 0)
        CAS_CUDA(ctx, cudaMemcpyAsync(jobs[j].row_digests, out.rows + PA.row_base[j],
                                      sizeof(uint64_t) * jobs[j].A.num_row, cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t j = 0; j < n; ++j) {
      jobs[j].digest = hd[(size_t)j];
      jobs[j].nnz_c = (int64_t)hn[(size_t)j];
      jobs[j].status = CAS_OK;
    }
    return CAS_OK;
  }();
  if (flp) cudaFreeAsync(flp, ctx->stream);
  if (bound) cudaFreeAsync(bound, ctx->stream);
  packed_free(ctx, PA);
  packed_free(ctx, PB);
  batch_out_free(ctx, out);
  return rc;
}

cas_status batch_per_call(cas_ctx* ctx, cas_accum accum, cas_job* jobs, int64_t n, cas_batch_stats& st) {
  using namespace cas;
  BatchOut out;
  int64_t* zero = nullptr;
  cas_status first = CAS_OK;
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(batch_out_alloc(ctx, n, 0, false, out));
    CAS_TRY(dev_alloc(ctx, (void**)&zero, sizeof(int64_t)));
    CAS_CUDA(ctx, cudaMemsetAsync(zero, 0, sizeof(int64_t), ctx->stream));
    int64_t max_rows = 0;
    for (int64_t j = 0; j < n; ++j)
      if (jobs[j].row_digests) max_rows = std::max(max_rows, jobs[j].A.num_row);
    uint64_t* rows = nullptr;
    if (max_rows > 0) CAS_TRY(dev_alloc(ctx, (void**)&rows, sizeof(uint64_t) * max_rows));
    for (int64_t j = 0; j < n; ++j) {
      cas_csr C{};
      C.on_device = 1;
      cas_status s = run_spgemm(ctx, accum, &jobs[j].A, &jobs[j].B, &C, nullptr);
      jobs[j].status = s;
      if (s != CAS_OK) {
        if (first == CAS_OK) first = s;
        continue;
      }
      jobs[j].flop = ctx->stats.flop;
      st.flop += ctx->stats.flop;
      st.nnz_c += C.num_nnz;
      st.h2d_bytes += ctx->stats.h2d_bytes;
      cas_status ds = digest_launch(ctx, C, 0, nullptr, zero, zero, out.digest + j, out.nnz + j,
                                    jobs[j].row_digests ? rows : nullptr);
      if (ds == CAS_OK && jobs[j].row_digests && C.num_row > 0)
        ds = cudaMemcpyAsync(jobs[j].row_digests, rows, sizeof(uint64_t) * C.num_row, cudaMemcpyDeviceToHost,
                             ctx->stream) == cudaSuccess ? CAS_OK : CAS_ERR_CUDA;
      cas_csr_free(ctx, &C);
      if (ds != CAS_OK) {
        jobs[j].status = ds;
        if (first == CAS_OK) first = ds;
      }
      st.waves++;
    }
    if (rows) CAS_CUDA(ctx, cudaFreeAsync(rows, ctx->stream));
    std::vector<unsigned long long> hd((size_t)n), hn((size_t)n);
    CAS_CUDA(ctx, cudaMemcpyAsync(hd.data(), out.digest, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(hn.data(), out.nnz, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t j = 0; j < n; ++j) {
      if (jobs[j].status != CAS_OK) continue;
      jobs[j].digest = hd[(size_t)j];
      jobs[j].nnz_c = (int64_t)hn[(size_t)j];
    }
    return first;
  }();
  if (zero) cudaFreeAsync(zero, ctx->stream);
  batch_out_free(ctx, out);
  return rc;
}


// CAS_BATCH_CONCURRENT: the jobs as in PER_CALL, on kBatchWorkers host
// threads with a context each (kept by the calling context).  The threads
// claim jobs from a shared counter, largest first by the estimate
// nnz(A) * nnz(B) / rows(B) (longest processing time first, so the jobs
// claimed last are short), and run them on their own streams: one job's host
// waits overlap the others' kernels, and small jobs' kernels, which leave
// most SMs idle, run side by side.  Each worker sizes its optional scratch
// (kept bitmaps, split rows) by 1 / kBatchWorkers of the free device memory;
// a job that still runs out of device memory beside the others is run again
// after them, alone, on the calling context.  Digests go into the calling
// context's per-job arrays; `ready` (recorded on its stream after they are
// cleared) orders the workers after that, and the calling stream waits for
// every worker's last kernel before they are read.
constexpr int kBatchWorkers = 4;

cas_status batch_concurrent(cas_ctx* ctx, cas_accum accum, cas_job* jobs, int64_t n, cas_batch_stats& st) {
  using namespace cas;
  const int nw = (int)std::min<int64_t>(kBatchWorkers, n);
  cas_tuning tun;
  cas_get_tuning(ctx, &tun);
  while ((int)ctx->batch_workers.size() < nw) {
    cas_ctx* w = nullptr;
    const cas_status s = cas_create(ctx->device, &w);
    if (s != CAS_OK) return set_err(ctx, s, "a batch worker's context could not be created");
    w->mem_share = 1.0 / kBatchWorkers;
    ctx->batch_workers.push_back(w);
  }
  std::vector<int64_t> order((size_t)n);
  std::vector<double> est((size_t)n);
  for (int64_t j = 0; j < n; ++j) {
    order[(size_t)j] = j;
    const cas_csr& B = jobs[j].B;
    est[(size_t)j] = (double)jobs[j].A.num_nnz * (double)B.num_nnz / (double)std::max<int64_t>(1, B.num_row);
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return est[(size_t)a] > est[(size_t)b]; });
  int64_t max_rows = 0;
  for (int64_t j = 0; j < n; ++j)
    if (jobs[j].row_digests) max_rows = std::max(max_rows, jobs[j].A.num_row);
  BatchOut out;
  CAS_TRY(batch_out_alloc(ctx, n, 0, false, out));
  cudaEvent_t ready = nullptr;
  CAS_CUDA(ctx, cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CAS_CUDA(ctx, cudaEventRecord(ready, ctx->stream));
  struct Tally {
    int64_t flop = 0, nnz = 0, runs = 0, launches = 0;
    double h2d = 0;
    cas_status first = CAS_OK;
    int64_t first_job = -1;
    std::string err;
    cudaEvent_t done = nullptr;
  };
  // one job on context w: its product, and its digest into the batch's arrays
  auto run_job = [&](cas_ctx* w, int64_t j, const int64_t* zero, uint64_t* rows, Tally& t) -> cas_status {
    cas_csr C{};
    C.on_device = 1;
    cas_status js = run_spgemm(w, accum, &jobs[j].A, &jobs[j].B, &C, nullptr);
    if (js != CAS_OK) return js;
    jobs[j].flop = w->stats.flop;
    t.flop += w->stats.flop;
    t.nnz += C.num_nnz;
    t.h2d += w->stats.h2d_bytes;
    js = digest_launch(w, C, 0, nullptr, zero, zero, out.digest + j, out.nnz + j, jobs[j].row_digests ? rows : nullptr);
    if (js == CAS_OK && jobs[j].row_digests && C.num_row > 0 &&
        cudaMemcpyAsync(jobs[j].row_digests, rows, sizeof(uint64_t) * C.num_row, cudaMemcpyDeviceToHost,
                        w->stream) != cudaSuccess)
      js = set_err(w, CAS_ERR_CUDA, "row digests of job %lld", (long long)j);
    cas_csr_free(w, &C);
    ++t.runs;
    return js;
  };
  // a worker's (or the calling context's) scratch for the digests
  auto job_scratch = [&](cas_ctx* w, int64_t** zero, uint64_t** rows) -> cas_status {
    CAS_TRY(dev_alloc(w, (void**)zero, sizeof(int64_t)));
    CAS_CUDA(w, cudaMemsetAsync(*zero, 0, sizeof(int64_t), w->stream));
    if (max_rows > 0) CAS_TRY(dev_alloc(w, (void**)rows, sizeof(uint64_t) * (size_t)max_rows));
    return CAS_OK;
  };
  std::vector<Tally> tally((size_t)nw + 1);  // the last: the calling context's retries
  std::atomic<int64_t> next{0};
  std::mutex retry_mu;
  std::vector<int64_t> retry;
  auto fail = [](Tally& t, cas_ctx* w, int64_t j, cas_status s) {
    if (t.first == CAS_OK) {
      t.first = s;
      t.first_job = j;
      t.err = w->err;
    }
  };
  auto work = [&](int wi) {
    cas_ctx* w = ctx->batch_workers[(size_t)wi];
    Tally& t = tally[(size_t)wi];
    cudaSetDevice(w->device);
    const int64_t l0 = w->launches;
    int64_t* zero = nullptr;
    uint64_t* rows = nullptr;
    cas_status s = cas_set_tuning(w, &tun);
    if (s == CAS_OK && cudaStreamWaitEvent(w->stream, ready, 0) != cudaSuccess)
      s = set_err(w, CAS_ERR_CUDA, "batch worker: wait for the batch's start");
    if (s == CAS_OK) s = job_scratch(w, &zero, &rows);
    if (s != CAS_OK) fail(t, w, -1, s);
    for (;;) {
      const int64_t i = next.fetch_add(1);
      if (i >= n) break;
      const int64_t j = order[(size_t)i];
      if (s != CAS_OK) {  // this worker cannot run jobs: the claimed one fails
        jobs[j].status = s;
        continue;
      }
      const cas_status js = run_job(w, j, zero, rows, t);
      if (js == CAS_ERR_OOM) {  // again after the others, alone
        std::lock_guard<std::mutex> lock(retry_mu);
        retry.push_back(j);
        continue;
      }
      jobs[j].status = js;
      if (js != CAS_OK) fail(t, w, j, js);
    }
    if (zero) cudaFreeAsync(zero, w->stream);
    if (rows) cudaFreeAsync(rows, w->stream);
    if (cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming) == cudaSuccess)
      cudaEventRecord(t.done, w->stream);
    t.launches = w->launches - l0;
  };
  std::vector<std::thread> threads;
  for (int wi = 0; wi < nw; ++wi) threads.emplace_back(work, wi);
  for (std::thread& th : threads) th.join();
  cudaEventDestroy(ready);
  for (int wi = 0; wi < nw; ++wi) {
    Tally& t = tally[(size_t)wi];
    if (t.done) {
      cudaStreamWaitEvent(ctx->stream, t.done, 0);
      cudaEventDestroy(t.done);
    }
  }
  if (!retry.empty()) {
    std::sort(retry.begin(), retry.end(), [&](int64_t a, int64_t b) { return est[(size_t)a] > est[(size_t)b]; });
    Tally& t = tally[(size_t)nw];  // its launches count on the calling context itself
    int64_t* zero = nullptr;
    uint64_t* rows = nullptr;
    cas_status s = job_scratch(ctx, &zero, &rows);
    for (const int64_t j : retry) {
      const cas_status js = s == CAS_OK ? run_job(ctx, j, zero, rows, t) : s;
      jobs[j].status = js;
      if (js != CAS_OK) fail(t, ctx, j, js);
    }
    if (zero) cudaFreeAsync(zero, ctx->stream);
    if (rows) cudaFreeAsync(rows, ctx->stream);
  }
  cas_status first = CAS_OK;
  for (Tally& t : tally) {
    st.flop += t.flop;
    st.nnz_c += t.nnz;
    st.h2d_bytes += t.h2d;
    st.waves += t.runs;
    ctx->launches += t.launches;
    if (first == CAS_OK && t.first != CAS_OK) {
      first = t.first;
      set_err(ctx, t.first, "batch job %lld: %s", (long long)t.first_job, t.err.c_str());
    }
  }
  std::vector<unsigned long long> hd((size_t)n), hn((size_t)n);
  CAS_CUDA(ctx, cudaMemcpyAsync(hd.data(), out.digest, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                ctx->stream));
  CAS_CUDA(ctx, cudaMemcpyAsync(hn.data(), out.nnz, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int64_t j = 0; j < n; ++j) {
    if (jobs[j].status != CAS_OK) continue;
    jobs[j].digest = hd[(size_t)j];
    jobs[j].nnz_c = (int64_t)hn[(size_t)j];
  }
  batch_out_free(ctx, out);
  return first;
}

}  // namespace

extern "C" {

cas_status cas_csr_digest(cas_ctx* ctx, const cas_csr* C, uint64_t* digest, uint64_t* row_digests) {
  if (!ctx || !C || !digest) return CAS_ERR_BAD_INPUT;
  CAS_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!C->on_device || C->col_bytes != 4)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "cas_csr_digest takes a device CSR with int32 columns");
  BatchOut out;
  int64_t* zero = nullptr;
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(batch_out_alloc(ctx, 1, C->num_row, row_digests != nullptr, out));
    CAS_TRY(dev_alloc(ctx, (void**)&zero, sizeof(int64_t)));
    CAS_CUDA(ctx, cudaMemsetAsync(zero, 0, sizeof(int64_t), ctx->stream));
    CAS_TRY(digest_launch(ctx, *C, 0, nullptr, zero, zero, out.digest, out.nnz, out.rows));
    unsigned long long h = 0;
    CAS_CUDA(ctx, cudaMemcpyAsync(&h, out.digest, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    if (row_digests && C->num_row > 0)
      CAS_CUDA(ctx, cudaMemcpyAsync(row_digests, out.rows, sizeof(uint64_t) * C->num_row, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *digest = h;
    return CAS_OK;
  }();
  if (zero) cudaFreeAsync(zero, ctx->stream);
  batch_out_free(ctx, out);
  return rc;
}

cas_status cas_batch_run(cas_ctx* ctx, cas_accum accum, cas_job* jobs, int64_t n, cas_batch_mode mode,
                         double wave_budget, cas_batch_stats* stats) {
  if (!ctx || (n > 0 && !jobs) || n < 0) return CAS_ERR_BAD_INPUT;
  if (accum != CAS_ACC_HASH && accum != CAS_ACC_HSERSC && accum != CAS_ACC_HYBACC)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "unknown accumulator %d", (int)accum);
  if (mode != CAS_BATCH_WAVES && mode != CAS_BATCH_PER_CALL && mode != CAS_BATCH_CONCURRENT)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "unknown batch mode %d", (int)mode);
  CAS_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaGetLastError();
  cas_batch_stats st{};
  if (n == 0) {
    if (stats) *stats = st;
    return CAS_OK;
  }
  const int vt = jobs[0].A.val_type;
  for (int64_t j = 0; j < n; ++j) {
    jobs[j].status = CAS_ERR_ABORTED;
    jobs[j].flop = jobs[j].nnz_c = 0;
    jobs[j].digest = 0;
  }
  for (int64_t j = 0; j < n; ++j) {
    const cas_csr& A = jobs[j].A;
    const cas_csr& B = jobs[j].B;
    cas_status s = basic_checks(ctx, &A, "A");
    if (s == CAS_OK) s = basic_checks(ctx, &B, "B");
    if (s == CAS_OK && (A.num_col != B.num_row || A.val_type != vt || B.val_type != vt || A.col_bytes != 4 ||
                        B.col_bytes != 4))
      s = set_err(ctx, CAS_ERR_BAD_INPUT, "job %lld: shapes, value types or column widths do not fit the batch",
                  (long long)j);
    if (s == CAS_OK && mode == CAS_BATCH_WAVES) {
      for (const cas_csr* M : {&A, &B})
        if (!M->on_device && (M->row_ptrs[0] != 0 || M->row_ptrs[M->num_row] != M->num_nnz))
          s = set_err(ctx, CAS_ERR_BAD_INPUT, "job %lld: row pointers do not span [0, num_nnz]", (long long)j);
    }
    if (s != CAS_OK) {
      jobs[j].status = s;
      return s;
    }
  }
  const int64_t launches0 = ctx->launches;
  cudaEvent_t e0, e1;
  CAS_CUDA(ctx, cudaEventCreate(&e0));
  CAS_CUDA(ctx, cudaEventCreate(&e1));
  CAS_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  const double budget = wave_budget > 0 ? wave_budget : 32.0 * (1ull << 30);
  cas_status rc = mode == CAS_BATCH_WAVES ? batch_waves(ctx, accum, jobs, n, budget, vt == CAS_VAL_F64 ? 8 : 4, st)
                  : mode == CAS_BATCH_PER_CALL ? batch_per_call(ctx, accum, jobs, n, st)
                                               : batch_concurrent(ctx, accum, jobs, n, st);
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  st.seconds = ms * 1e-3;
  st.kernel_launches = ctx->launches - launches0;
  for (int64_t j = 0; j < n; ++j) st.jobs_ok += jobs[j].status == CAS_OK;
  if (stats) *stats = st;
  return rc;
}

}  // extern "C"
