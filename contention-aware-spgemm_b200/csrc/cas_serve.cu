// Serving: a request loop with continuous batching (declared in
// include/casgemm.h).  Part of the cas_api.cu translation unit.
//
// `slots` worker threads each own a context (stream and auxiliary streams)
// on the device.  Requests queue in arrival order; a worker takes the head
// of the queue when the head's reserved device bytes fit beside those of the
// requests already running, runs it with the product pipeline, and frees
// its reservation.  Several requests are therefore on the device at once,
// and a request that arrives while others run starts as soon as a slot and
// its memory are free, without waiting for the running ones to drain.  Only
// the head is ever admitted, so a large request is not overtaken forever.
// A request whose bound is larger than the whole budget runs as row chunks
// that each fit (rows of C are independent); its digest is the sum of the
// chunks' digests, which the row offsets of the digest make exact.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

struct ServeReq {
  int64_t id = 0;
  cas_csr A{}, B{};
  std::vector<int64_t> cuts;  // row chunk boundaries
  std::vector<int64_t> a_rp;  // device A split into chunks: A's row pointers, copied at submission
  int64_t flop = 0;
  cas_result res{};
  bool done = false;
};

double host_csr_device_bytes(const cas_csr& M) {
  return 8.0 * (double)(M.num_row + 1) + (4.0 + (M.val_type == CAS_VAL_F64 ? 8.0 : 4.0)) * (double)M.num_nnz;
}

// Row products of a device request (sum over A_i of |B_k|) for its memory
// bound, and a check of its structure: row pointers that start at 0, end at
// nnz and do not decrease, columns inside B.  `bad` becomes nonzero on a
// violation (the row products are then meaningless).
__global__ void k_serve_row_products(int64_t m, int64_t nnz, const int64_t* __restrict__ arp,
                                     const int32_t* __restrict__ acol, int64_t brows, const int64_t* __restrict__ brp,
                                     int64_t* __restrict__ out, int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (arp[0] != 0 || arp[m] != nnz)) atomicOr(bad, 1);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += warps) {
    const int64_t s = arp[i], e = arp[i + 1];
    if (e < s) {
      if (lane == 0) atomicOr(bad, 2);
      continue;
    }
    long long p = 0;
    for (int64_t k = s + lane; k < e; k += 32) {
      const int32_t c = acol[k];
      if (c < 0 || c >= brows) {
        atomicOr(bad, 4);
        continue;
      }
      p += brp[c + 1] - brp[c];
    }
    p = cas::warp_sum(p);
    if (lane == 0) out[i] = p;
  }
}

// Row pointers of rows [r0, r1) of a device CSR, rebased to start at 0.
__global__ void k_serve_rebase(int64_t n, const int64_t* __restrict__ src, int64_t base, int64_t* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i] - base;
}

}  // namespace

struct cas_server {
  cas_server_opts opts{};
  int device = 0;
  std::mutex mu;
  std::mutex submit_mu;              // device requests: one sizing pass at a time
  cudaStream_t submit_stream = nullptr;
  std::condition_variable cv;
  std::deque<ServeReq*> pending;
  std::unordered_map<int64_t, ServeReq*> reqs;
  int64_t next_id = 1;
  double inflight_bytes = 0;
  int inflight = 0;
  bool stopping = false;
  cas_server_stats stats{};
  std::vector<std::thread> workers;
  std::vector<cas_ctx*> ctxs;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// Runs one request on a slot's context: each row chunk through the pipeline,
// its digest folded in on the device, C copied out when the caller keeps it.
cas_status serve_execute(cas_server* srv, cas_ctx* ctx, ServeReq* r) {
  using namespace cas;
  const cas_csr& A = r->A;
  const bool f64 = A.val_type == CAS_VAL_F64;
  unsigned long long *d_digest = nullptr, *d_nnz = nullptr;
  int64_t* zero = nullptr;
  std::vector<int64_t> out_rp;
  std::vector<int32_t> out_col;
  std::vector<char> out_val;
  const bool keep = srv->opts.keep_output != 0;
  if (keep) out_rp.push_back(0);
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(dev_alloc(ctx, (void**)&d_digest, sizeof(unsigned long long)));
    CAS_TRY(dev_alloc(ctx, (void**)&d_nnz, sizeof(unsigned long long)));
    CAS_TRY(dev_alloc(ctx, (void**)&zero, sizeof(int64_t)));
    CAS_CUDA(ctx, cudaMemsetAsync(d_digest, 0, sizeof(unsigned long long), ctx->stream));
    CAS_CUDA(ctx, cudaMemsetAsync(d_nnz, 0, sizeof(unsigned long long), ctx->stream));
    CAS_CUDA(ctx, cudaMemsetAsync(zero, 0, sizeof(int64_t), ctx->stream));
    std::vector<int64_t> rp;
    int64_t* d_rp = nullptr;  // device A in chunks: the chunk's rebased row pointers
    struct RpFree {
      cas_ctx* c;
      int64_t** p;
      ~RpFree() {
        if (*p) cudaFreeAsync(*p, c->stream);
      }
    } rp_free{ctx, &d_rp};
    for (size_t k = 0; k + 1 < r->cuts.size(); ++k) {
      const int64_t r0 = r->cuts[k], r1 = r->cuts[k + 1];
      cas_csr Ac = A;
      if (r->cuts.size() > 2 && A.on_device) {  // a device row slice: row pointers rebased on the device
        const int64_t base = r->a_rp[(size_t)r0];
        if (!d_rp) CAS_TRY(dev_alloc(ctx, (void**)&d_rp, sizeof(int64_t) * (size_t)(A.num_row + 1)));
        k_serve_rebase<<<grid_for(r1 - r0 + 1, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(
            r1 - r0 + 1, A.row_ptrs + r0, base, d_rp);
        CAS_TRY(check_launch(ctx, "k_serve_rebase"));
        Ac.num_row = r1 - r0;
        Ac.num_nnz = r->a_rp[(size_t)r1] - base;
        Ac.row_ptrs = d_rp;
        Ac.cols = static_cast<int32_t*>(A.cols) + base;
        Ac.rats = static_cast<char*>(A.rats) + (f64 ? 8 : 4) * base;
      } else if (r->cuts.size() > 2) {  // a host row slice whose row pointers start at 0
        rp.resize((size_t)(r1 - r0 + 1));
        for (int64_t i = r0; i <= r1; ++i) rp[(size_t)(i - r0)] = A.row_ptrs[i] - A.row_ptrs[r0];
        Ac.num_row = r1 - r0;
        Ac.num_nnz = rp.back();
        Ac.row_ptrs = rp.data();
        Ac.cols = static_cast<int32_t*>(A.cols) + A.row_ptrs[r0];
        Ac.rats = static_cast<char*>(A.rats) + (f64 ? 8 : 4) * A.row_ptrs[r0];
      }
      cas_csr C{};
      C.on_device = 1;
      CAS_TRY(run_spgemm(ctx, (cas_accum)srv->opts.accum, &Ac, &r->B, &C, nullptr));
      r->res.flop += ctx->stats.flop;
      cas_status ds = digest_launch(ctx, C, r0, nullptr, zero, zero, d_digest, d_nnz, nullptr);
      if (ds == CAS_OK && keep && C.num_row > 0) {
        const size_t base = out_col.size();
        std::vector<int64_t> crp((size_t)C.num_row + 1);
        out_col.resize(base + (size_t)C.num_nnz);
        out_val.resize((base + (size_t)C.num_nnz) * 8);
        if (cudaMemcpyAsync(crp.data(), C.row_ptrs, sizeof(int64_t) * crp.size(), cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess ||
            cudaMemcpyAsync(out_col.data() + base, C.cols, sizeof(int32_t) * C.num_nnz, cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess ||
            cudaMemcpyAsync(out_val.data() + base * 8, C.rats, 8 * (size_t)C.num_nnz, cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
          ds = set_err(ctx, CAS_ERR_CUDA, "copy of C to the host failed");
        for (int64_t i = 1; i <= C.num_row; ++i) out_rp.push_back((int64_t)base + crp[(size_t)i]);
      }
      cas_csr_free(ctx, &C);
      CAS_TRY(ds);
    }
    unsigned long long h[2] = {0, 0};
    CAS_CUDA(ctx, cudaMemcpyAsync(&h[0], d_digest, sizeof(h[0]), cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(&h[1], d_nnz, sizeof(h[1]), cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    r->res.digest = h[0];
    r->res.nnz_c = (int64_t)h[1];
    return CAS_OK;
  }();
  void* ps[] = {d_digest, d_nnz, zero};
  for (void* p : ps)
    if (p) cudaFreeAsync(p, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  if (rc == CAS_OK && keep) {
    cas_csr& C = r->res.C;
    C.num_row = A.num_row;
    C.num_col = r->B.num_col;
    C.num_nnz = (int64_t)out_col.size();
    C.col_bytes = 4;
    C.val_type = A.val_type;
    C.on_device = 0;
    C.owned = 1;
    C.row_ptrs = static_cast<int64_t*>(malloc(sizeof(int64_t) * out_rp.size()));
    C.cols = malloc(sizeof(int32_t) * (out_col.size() > 0 ? out_col.size() : 1));
    C.rats = malloc(out_val.size() > 0 ? out_val.size() : 8);
    if (!C.row_ptrs || !C.cols || !C.rats) {
      free(C.row_ptrs); free(C.cols); free(C.rats);
      memset(&C, 0, sizeof(C));
      return CAS_ERR_OOM;
    }
    memcpy(C.row_ptrs, out_rp.data(), sizeof(int64_t) * out_rp.size());
    memcpy(C.cols, out_col.data(), sizeof(int32_t) * out_col.size());
    memcpy(C.rats, out_val.data(), out_val.size());
  }
  return rc;
}

void serve_worker(cas_server* srv, int slot) {
  cas_ctx* ctx = srv->opts.dry_run ? nullptr : srv->ctxs[(size_t)slot];
  if (ctx) cudaSetDevice(srv->device);
  for (;;) {
    ServeReq* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      srv->cv.wait(lk, [&] {
        if (!srv->pending.empty())
          return srv->inflight_bytes + srv->pending.front()->res.bound <= srv->opts.mem_budget ||
                 srv->inflight == 0;
        return srv->stopping;
      });
      if (srv->pending.empty()) return;
      r = srv->pending.front();
      srv->pending.pop_front();
      srv->inflight_bytes += r->res.bound;
      srv->inflight++;
      srv->stats.max_inflight = std::max(srv->stats.max_inflight, srv->inflight);
      srv->stats.max_inflight_bytes = std::max(srv->stats.max_inflight_bytes, srv->inflight_bytes);
      r->res.t_admit = srv->now();
    }
    cas_status st;
    if (ctx) {
      st = serve_execute(srv, ctx, r);
    } else {
      std::this_thread::sleep_for(std::chrono::nanoseconds((int64_t)(r->res.bound * srv->opts.dry_run_ns_per_byte)));
      r->res.flop = r->flop;
      st = CAS_OK;
    }
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->inflight_bytes -= r->res.bound;
      srv->inflight--;
      r->res.status = st;
      r->res.t_done = srv->now();
      r->done = true;
      if (st == CAS_OK) srv->stats.completed++;
      else srv->stats.failed++;
    }
    srv->cv.notify_all();
  }
}

}  // namespace

extern "C" {

cas_status cas_serve_create(int device, const cas_server_opts* opts, cas_server** out) {
  if (!out) return CAS_ERR_BAD_INPUT;
  *out = nullptr;
  cas_server* srv = new (std::nothrow) cas_server();
  if (!srv) return CAS_ERR_OOM;
  if (opts) srv->opts = *opts;
  if (srv->opts.slots <= 0) srv->opts.slots = 4;
  if (srv->opts.mem_budget <= 0) srv->opts.mem_budget = 60e9;
  if (srv->opts.accum < CAS_ACC_HASH || srv->opts.accum > CAS_ACC_HYBACC) {
    delete srv;
    return CAS_ERR_BAD_INPUT;
  }
  srv->device = device;
  if (!srv->opts.dry_run) {
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&srv->submit_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete srv;
      return CAS_ERR_CUDA;
    }
    for (int i = 0; i < srv->opts.slots; ++i) {
      cas_ctx* c = nullptr;
      const cas_status st = cas_create(device, &c);
      if (st != CAS_OK) {
        for (cas_ctx* x : srv->ctxs) cas_destroy(x);
        cudaStreamDestroy(srv->submit_stream);
        delete srv;
        return st;
      }
      srv->ctxs.push_back(c);
    }
  }
  for (int i = 0; i < srv->opts.slots; ++i) srv->workers.emplace_back(serve_worker, srv, i);
  *out = srv;
  return CAS_OK;
}

// Row products of a device request, with its structure checked on the
// device; fills rowp (m entries) and, when keep_rp, A's row pointers.
static cas_status serve_device_rows(cas_server* srv, const cas_csr* A, const cas_csr* B, std::vector<int64_t>& rowp,
                                    std::vector<int64_t>* a_rp) {
  std::lock_guard<std::mutex> lk(srv->submit_mu);
  if (cudaSetDevice(srv->device) != cudaSuccess) return CAS_ERR_CUDA;
  const int64_t m = A->num_row;
  cudaStream_t s = srv->submit_stream;
  int64_t* d_out = nullptr;
  int* d_bad = nullptr;
  int bad = 0;
  cas_status rc = CAS_OK;
  if (cudaMallocAsync((void**)&d_out, sizeof(int64_t) * (size_t)(m > 0 ? m : 1), s) != cudaSuccess ||
      cudaMallocAsync((void**)&d_bad, sizeof(int), s) != cudaSuccess) {
    rc = CAS_ERR_OOM;
  } else {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, srv->device);
    cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    const int64_t blocks = std::min<int64_t>((m * 32 + 255) / 256 + 1, (int64_t)sms * 8);
    k_serve_row_products<<<(unsigned)blocks, 256, 0, s>>>(m, A->num_nnz, A->row_ptrs,
                                                          static_cast<const int32_t*>(A->cols), B->num_row,
                                                          B->row_ptrs, d_out, d_bad);
    rowp.resize((size_t)m);
    if (a_rp) a_rp->resize((size_t)m + 1);
    if (cudaGetLastError() != cudaSuccess ||
        (m > 0 && cudaMemcpyAsync(rowp.data(), d_out, sizeof(int64_t) * (size_t)m, cudaMemcpyDeviceToHost, s) !=
                      cudaSuccess) ||
        (a_rp && cudaMemcpyAsync(a_rp->data(), A->row_ptrs, sizeof(int64_t) * (size_t)(m + 1),
                                 cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      rc = CAS_ERR_CUDA;
    else if (bad)
      rc = CAS_ERR_BAD_INPUT;
  }
  if (d_out) cudaFreeAsync(d_out, s);
  if (d_bad) cudaFreeAsync(d_bad, s);
  cudaStreamSynchronize(s);
  if (rc == CAS_ERR_CUDA) cudaGetLastError();
  return rc;
}

cas_status cas_serve_submit(cas_server* srv, const cas_csr* A, const cas_csr* B, int64_t* id) {
  if (!srv || !A || !B || !id) return CAS_ERR_BAD_INPUT;
  if (basic_checks(nullptr, A, "A") != CAS_OK || basic_checks(nullptr, B, "B") != CAS_OK) return CAS_ERR_BAD_INPUT;
  const bool dev = A->on_device != 0;
  if (B->on_device != A->on_device || A->col_bytes != 4 || B->col_bytes != 4 || A->num_col != B->num_row ||
      A->val_type != B->val_type || (dev && srv->opts.dry_run))
    return CAS_ERR_BAD_INPUT;
  if (!dev)
    for (const cas_csr* M : {A, B})
      if (M->row_ptrs[0] != 0 || M->row_ptrs[M->num_row] != M->num_nnz) return CAS_ERR_BAD_INPUT;
  ServeReq* r = new (std::nothrow) ServeReq();
  if (!r) return CAS_ERR_OOM;
  r->A = *A;
  r->B = *B;
  // row products: on the host for host operands, on the device (and the
  // structure checked there) for resident ones
  std::vector<int64_t> rowp((size_t)A->num_row);
  if (dev) {
    std::vector<int64_t> a_rp;
    const cas_status st = serve_device_rows(srv, A, B, rowp, &a_rp);
    if (st != CAS_OK) {
      delete r;
      return st;
    }
    r->a_rp.swap(a_rp);
  } else {
    const int32_t* acol = static_cast<const int32_t*>(A->cols);
    for (int64_t i = 0; i < A->num_row; ++i) {
      int64_t p = 0;
      for (int64_t k = A->row_ptrs[i]; k < A->row_ptrs[i + 1]; ++k) {
        const int32_t c = acol[k];
        if (c < 0 || c >= B->num_row) {
          delete r;
          return CAS_ERR_BAD_INPUT;
        }
        p += B->row_ptrs[c + 1] - B->row_ptrs[c];
      }
      rowp[(size_t)i] = p;
    }
  }
  // per-row bound: 12 bytes per possible entry of C, 40 per row (the row
  // pointers of A and C and the pipeline's per-row scratch) and, for host
  // operands, the row's share of A's device copy; B's copy is fixed.
  // Resident operands are the caller's memory and are not counted.
  const double fixed = 16.0 + (dev ? 0.0 : host_csr_device_bytes(*B));
  const double budget = srv->opts.mem_budget;
  const double ebytes = dev ? 0.0 : 4.0 + (A->val_type == CAS_VAL_F64 ? 8.0 : 4.0);
  double total = fixed, chunk = fixed, chunk_max = 0;
  r->cuts.push_back(0);
  std::vector<double> rowb((size_t)A->num_row);
  const int64_t* arp = dev ? r->a_rp.data() : A->row_ptrs;
  for (int64_t i = 0; i < A->num_row; ++i) {
    const int64_t p = rowp[(size_t)i];
    r->flop += p;
    rowb[(size_t)i] = 12.0 * (double)std::min<int64_t>(p, B->num_col) + 40.0 + ebytes * (double)(arp[i + 1] - arp[i]);
    total += rowb[(size_t)i];
  }
  r->res.chunks = 1;
  if (total <= budget) {
    r->cuts.push_back(A->num_row);
    r->res.bound = total;
  } else {
    // row chunks whose bound (with B's copy) fits the budget
    for (int64_t i = 0; i < A->num_row; ++i) {
      if (chunk + rowb[(size_t)i] > budget && i > r->cuts.back()) {
        chunk_max = std::max(chunk_max, chunk);
        r->cuts.push_back(i);
        chunk = fixed;
      }
      chunk += rowb[(size_t)i];
    }
    chunk_max = std::max(chunk_max, chunk);
    r->cuts.push_back(A->num_row);
    r->res.chunks = (int32_t)(r->cuts.size() - 1);
    r->res.bound = chunk_max;
  }
  if (r->res.chunks == 1) std::vector<int64_t>().swap(r->a_rp);
  std::lock_guard<std::mutex> lk(srv->mu);
  r->id = srv->next_id++;
  r->res.t_submit = srv->now();
  srv->reqs[r->id] = r;
  srv->stats.submitted++;
  if (r->res.bound > budget) {  // one row with B's copy is already over the budget
    r->res.status = CAS_ERR_REJECTED;
    r->res.t_admit = r->res.t_done = r->res.t_submit;
    r->done = true;
    srv->stats.failed++;
  } else {
    if (r->res.chunks > 1) srv->stats.chunked++;
    srv->pending.push_back(r);
  }
  *id = r->id;
  srv->cv.notify_all();
  return CAS_OK;
}

cas_status cas_serve_poll(cas_server* srv, int64_t id, cas_result* out) {
  return cas_serve_wait(srv, id, 0.0, out);
}

cas_status cas_serve_wait(cas_server* srv, int64_t id, double timeout_s, cas_result* out) {
  if (!srv || !out) return CAS_ERR_BAD_INPUT;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return CAS_ERR_BAD_INPUT;
  ServeReq* r = it->second;
  if (timeout_s < 0) {
    srv->cv.wait(lk, [&] { return r->done; });
  } else if (!srv->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; })) {
    return CAS_ERR_TIMEOUT;
  }
  *out = r->res;
  srv->reqs.erase(it);
  delete r;
  return CAS_OK;
}

cas_status cas_serve_stats(cas_server* srv, cas_server_stats* out) {
  if (!srv || !out) return CAS_ERR_BAD_INPUT;
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->stats;
  return CAS_OK;
}

double cas_serve_clock(const cas_server* srv) { return srv ? srv->now() : 0.0; }

void cas_serve_destroy(cas_server* srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stopping = true;
  }
  srv->cv.notify_all();
  for (std::thread& t : srv->workers) t.join();
  for (cas_ctx* c : srv->ctxs) cas_destroy(c);
  if (srv->submit_stream) cudaStreamDestroy(srv->submit_stream);
  for (auto& kv : srv->reqs) {
    cas_csr& C = kv.second->res.C;
    if (C.owned && !C.on_device) {
      free(C.row_ptrs);
      free(C.cols);
      free(C.rats);
    }
    delete kv.second;
  }
  delete srv;
}

}  // extern "C"
