// casgemm C ABI and host orchestration (declarations in include/casgemm.h).
//
// One call of cas_spgemm runs the four phases of the reference's drivers
// (src/ams_hybaccspgemm.c:36-215) on the context's stream:
//   INIT  input check, k_flp (row products, totals, symbolic bin histogram),
//         symbolic bin lists
//   SYMB  symbolic kernels per bin (bins run concurrently on auxiliary
//         streams), scan of the counts into C's row pointers
//   MGMT  allocation of C, numeric bin lists
//   NUMC  numeric kernels per bin
// Each phase boundary is a CUDA event; the phase times are what cas_runtime
// reports, like the reference's runtime_t.  The host waits three times per
// call, each to size the next phase (bin counts, nnz(C)).
#include <cuda_runtime.h>

#include <immintrin.h>
#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "casgemm.h"
#include "cas_kernels.cu"

namespace {

constexpr int kAux = 4;          // auxiliary streams for concurrent bins
constexpr int kMaxOutBlocks = 64;  // row blocks of a C returned in host memory, at most
constexpr double kOutBlockMin = double(1ull << 30);    // host C under this: one block
constexpr double kOutBlockBytes = double(2ull << 30);  // else a block per this many bytes of C
constexpr int kCountSlots = 256; // device/pinned counter block
constexpr int kMiscWords = 8;    // pinned words of other small results

// Layout of the counter block (unsigned long long slots).
constexpr int kSlotSymb = 0;     // [0, 9)   symbolic bin counts
constexpr int kSlotNumc = 10;    // [10, 23) numeric bin counts
constexpr int kSlotTotals = 24;  // [24]    products, [25] max row products
constexpr int kSlotCursor = 28;  // [28, 41) bin cursors
constexpr int kSlotNnz = 44;     // [44]    nnz(C) from the scan
constexpr int kSlotCheck = 48;   // [48, 52) input check flags
constexpr int kSlotBinSums = 64; // [64, 103) per numeric bin: products, nnz(C), nnz(A)
constexpr int kSlotOvf = 110;    // [110]   rows handed to the radix-sort ESC kernel
constexpr int kSlotFused = 112;  // [112, 116) fused rows: count, products, output bound, nnz(A); [116] ticket
constexpr int kSlotHeavy = 128;  // [128, 176) dense rows per size class
constexpr int kSlotHeavyCur = 176;  // [176, 224) their cursors
constexpr size_t kStageBytes = size_t(64) << 20;  // pinned staging chunk for host copies
constexpr double kSavedBitmapBytes = 8.0 * (1ull << 30);  // heavy-row bitmaps kept between the phases

}  // namespace

struct cas_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kAux] = {};
  cudaEvent_t ev_phase[5] = {};
  cudaEvent_t ev_symb[2][cas::kSymbBins] = {};
  cudaEvent_t ev_numc[2][cas::kNumcBins] = {};
  cudaEvent_t ev_ovf[2] = {};
  bool profile = false;
  bool fuse = true;                        // fused ESC rows (no symbolic pass) in cas_spgemm
  int fused_lo = (int)cas::kFusedLo;       // fused rows: more products than this (up to kFusedHi)
  bool heavy_split = true;                 // dense rows of 2^17 products or more split across blocks
  int bin_order = 1;                       // 1: contended bins launched first; 0: interleaved with the ESC bins
  int esc_form = 2;                        // bucketed ESC of rows over 4096 products (fused rows included):
                                           // 1 index form (k_numc_esc_idx), 0 k_numc_esc_msd, 2 the index
                                           // form with the keys in registers between its two key passes
  int esc_max = 8192;                      // ESC rows: at most this many products
  int hash_max = 4096;                     // hash rows: at most this many distinct columns
  int out_blocks = 0;                      // C in host memory: row blocks (0: by C's size)
  double mem_share = 1.0;                  // share of the free device memory this context sizes
                                           // its optional scratch by (a batch worker's: 1 / workers)
  double acc_thres = 2.0;
  cudaEvent_t ev_fused[2] = {};
  cudaStream_t copy_stream = nullptr;      // copies of finished row blocks of a host C
  std::vector<cas_ctx*> batch_workers;     // contexts of CAS_BATCH_CONCURRENT's threads
  std::string err;
  cas_stats stats{};
  int64_t launches = 0;
  cas::DevStatus* d_status = nullptr;
  unsigned long long* d_counts = nullptr;
  unsigned long long* h_counts = nullptr;  // pinned mirror
  cas::DevStatus* h_status = nullptr;      // pinned mirror
  unsigned long long* h_misc = nullptr;    // pinned words for other small results
  // the mirrors' device-side addresses (the device writes them by k_fetch_words)
  unsigned long long* h_counts_dev = nullptr;
  unsigned long long* h_status_dev = nullptr;
  unsigned long long* h_misc_dev = nullptr;
  void* h_stage[3] = {};                   // pinned staging for large host copies
  cudaEvent_t ev_stage[3] = {};
  // host blocks of returned C arrays: capacity of every live block this
  // context allocated, and the released ones kept for reuse
  std::unordered_map<void*, size_t> host_blocks;
  std::vector<std::pair<void*, size_t>> host_free;
  // cached blocks registered with CUDA, which copies into them by DMA
  // directly; registration is turned off after it fails once
  std::unordered_set<void*> host_pinned;
  bool host_pin_off = false;
  double d2h_direct = 0;  // bytes the current call copied into registered blocks
  size_t host_free_bytes = 0;
};

namespace {

using cas::Csr;

cas_status set_err(cas_ctx* ctx, cas_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return st;
}

#define CAS_CUDA(ctx, call)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      return set_err(ctx, e_ == cudaErrorMemoryAllocation ? CAS_ERR_OOM : CAS_ERR_CUDA,      \
                     "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                        \
  } while (0)

#define CAS_TRY(x)                      \
  do {                                  \
    cas_status s_ = (x);                \
    if (s_ != CAS_OK) return s_;        \
  } while (0)

cas_status check_launch(cas_ctx* ctx, const char* what) {
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, CAS_ERR_CUDA, "launch of %s failed: %s (stream %p)", what, cudaGetErrorString(e),
                   (void*)ctx->stream);
  return CAS_OK;
}

const char* dev_err_name(int code) {
  switch (code) {
    case cas::kDevRowOverflow: return "a row produced more entries than its symbolic count";
    case cas::kDevRowUnderflow: return "a row produced fewer entries than its symbolic count";
    case cas::kDevCapacity: return "a row exceeded the shared-memory capacity of its kernel";
    case cas::kDevTableFull: return "a shared-memory hash table ran out of slots";
    case cas::kDevBadIndex: return "a column index is outside the matrix";
    default: return "unknown device error";
  }
}

// n words (8 bytes each) from device memory into a pinned mirror, written
// by a one-block kernel on s through the mirror's device-side address
// (mirror_dev); the caller synchronises s before reading the mirror.
static_assert(sizeof(cas::DevStatus) % 8 == 0, "the status is fetched in 8-byte words");
cas_status fetch_words(cas_ctx* ctx, unsigned long long* mirror_dev, const void* src, int n, cudaStream_t s) {
  cas::k_fetch_words<<<1, 256, 0, s>>>(mirror_dev, static_cast<const unsigned long long*>(src), n);
  return check_launch(ctx, "k_fetch_words");
}

cas_status check_status(cas_ctx* ctx) {
  CAS_TRY(fetch_words(ctx, ctx->h_status_dev, ctx->d_status, (int)(sizeof(cas::DevStatus) / 8), ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->h_status->err != 0) {
    return set_err(ctx, CAS_ERR_DEVICE, "device check failed in kernel %d at row %lld: %s", ctx->h_status->kernel,
                   (long long)ctx->h_status->row, dev_err_name(ctx->h_status->err));
  }
  return CAS_OK;
}

template <typename K>
cas_status allow_smem(cas_ctx* ctx, K kernel, size_t bytes) {
  CAS_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return CAS_OK;
}

// ------------------------------------------------ kernel shapes and memory
template <int BLOCK, int TBITS, int SEGCAP>
constexpr size_t smem_symb_hash() { return (size_t(1) << TBITS) * 4 + SEGCAP + sizeof(cas::StageB<double>); }
template <int BLOCK>
constexpr size_t smem_symb_dense() { return size_t(cas::kDenseChunkBits / 32) * 4 + sizeof(cas::Stage<double>); }
template <int BLOCK, int CAP, typename VIn>
constexpr size_t smem_numc_esc() {
  return size_t(CAP) * 16 + size_t(CAP) * sizeof(typename cas::Acc<VIn>::T) + sizeof(cas::SortScratch<BLOCK>) +
         sizeof(cas::Stage<VIn>);
}
template <int BLOCK, int TBITS, typename VIn>
constexpr size_t smem_numc_hash() {
  return (size_t(1) << TBITS) * (4 + sizeof(typename cas::Acc<VIn>::T)) + (size_t(1) << (TBITS - 1)) * 8 +
         sizeof(cas::SortScratch<BLOCK>) + sizeof(cas::Stage<VIn>);
}
template <int BLOCK, typename VIn>
constexpr size_t smem_numc_dense() {
  return size_t(cas::kRankCols / 32) * 4 + size_t(cas::kRankCols / 256) * 4 + size_t(cas::kRankCols / 32) * 2 +
         sizeof(cas::Stage<VIn>);
}

template <int CAP, int NBB, typename VIn>
constexpr size_t smem_numc_esc_msd() {
  return size_t(CAP) * (sizeof(typename cas::Acc<VIn>::T) + 4) + (size_t(1) << NBB) * 2 + size_t(CAP / 32) * 4 +
         ((size_t(CAP) + 15) & ~size_t(15)) + sizeof(cas::StageB<VIn>);
}

// index form: column, product index and place per product, padded chunk counts and head masks
template <int CAP, int NBB, typename VIn>
constexpr size_t smem_numc_esc_idx() {
  return size_t(CAP) * 8 + (size_t(1) << NBB) * 2 + size_t((CAP / 32 + 3) & ~3) * 8 +
         ((size_t(CAP) + 15) & ~size_t(15)) + sizeof(cas::StageB<VIn>);
}

// symbolic hash shape of each symbolic bin: threads, log2(table slots), byte
// table capacity (shared memory allows 3 CTAs per SM for the 16 Ki table)
#define CAS_SYMB_SHAPES(X)        \
  X(kSB_H1K, 128, 10, 1024)       \
  X(kSB_H2K, 128, 11, 2048)       \
  X(kSB_H4K, 256, 12, 4096)       \
  X(kSB_H8K, 256, 13, 4096)       \
  X(kSB_H16K, 256, 14, 8192)      \
  X(kSB_H32K, 512, 15, 16384)

// bucketed ESC shape of each ESC bin: capacity and log2(bucket count), two to
// four products per bucket; shared memory allows 8, 7, 4, 3, 3, 2, 1 CTAs of
// 256 threads per SM for the seven bins
#define CAS_ESC_SHAPES(X) \
  X(kNB_E1K, 1024, 9)   \
  X(kNB_E2K, 2048, 9)   \
  X(kNB_E3K, 3072, 10)  \
  X(kNB_E4K, 4096, 10)  \
  X(kNB_E5K, 4800, 11)  \
  X(kNB_E6K, 6144, 11)  \
  X(kNB_E8K, 8192, 11)

template <typename VIn>
cas_status setup_numc_kernels(cas_ctx* ctx) {
  using namespace cas;
#define CAS_SETUP_ESC(bin, CAP, NBB)                                                               \
  CAS_TRY(allow_smem(ctx, k_numc_esc_msd<256, CAP, NBB, VIn>, smem_numc_esc_msd<CAP, NBB, VIn>())); \
  if constexpr (CAP > 4096) CAS_TRY(allow_smem(ctx, k_numc_esc_idx<256, CAP, NBB, VIn>, smem_numc_esc_idx<CAP, NBB, VIn>())); \
  if constexpr (CAP > 4096 && CAP <= 6144)                                                         \
    CAS_TRY(allow_smem(ctx, k_numc_esc_idx<256, CAP, NBB, VIn, false, true>, smem_numc_esc_idx<CAP, NBB, VIn>()));
  CAS_ESC_SHAPES(CAS_SETUP_ESC)
#undef CAS_SETUP_ESC
  CAS_TRY(allow_smem(ctx, k_numc_esc_msd<256, (int)kFusedHi, 11, VIn, true>,
                     smem_numc_esc_msd<(int)kFusedHi, 11, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_esc_idx<256, (int)kFusedHi, 11, VIn, true>,
                     smem_numc_esc_idx<(int)kFusedHi, 11, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_esc_idx<256, (int)kFusedHi, 11, VIn, true, true>,
                     smem_numc_esc_idx<(int)kFusedHi, 11, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_esc_overflow<1024, 8192, VIn>, smem_numc_esc<1024, 8192, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_hash<256, 9, VIn>, smem_numc_hash<256, 9, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_hash<256, 11, VIn>, smem_numc_hash<256, 11, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_hash<512, 13, VIn>, smem_numc_hash<512, 13, VIn>()));
  CAS_TRY(allow_smem(ctx, k_numc_dense<512, VIn>, smem_numc_dense<512, VIn>()));
  CAS_TRY(allow_smem(ctx, k_dense_setup<512, VIn>, smem_numc_dense<512, VIn>()));
  CAS_TRY(allow_smem(ctx, k_dense_acc<512, VIn>, smem_numc_dense<512, VIn>()));
  return CAS_OK;
}

cas_status setup_kernels(cas_ctx* ctx) {
  using namespace cas;
#define CAS_SETUP_SYMB(bin, BLK, TB, SEG) CAS_TRY(allow_smem(ctx, k_symb_hash<BLK, TB, SEG>, smem_symb_hash<BLK, TB, SEG>()));
  CAS_SYMB_SHAPES(CAS_SETUP_SYMB)
#undef CAS_SETUP_SYMB
  CAS_TRY(allow_smem(ctx, k_symb_dense<512>, smem_symb_dense<512>()));
  CAS_TRY(allow_smem(ctx, k_heavy_bits<512>, smem_symb_dense<512>()));
  CAS_TRY(setup_numc_kernels<double>(ctx));
  CAS_TRY(setup_numc_kernels<int32_t>(ctx));
  return CAS_OK;
}

int grid_for(int64_t items, int block, int cap) {
  int64_t g = (items + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// ------------------------------------------------------- device matrices
struct DevMat {
  Csr csr{};
  int64_t nnz = 0;
  int vt = CAS_VAL_F64;
  std::vector<void*> owned;  // temporaries allocated for a host input
};

cas_status free_owned(cas_ctx* ctx, DevMat& m) {
  for (void* p : m.owned) CAS_CUDA(ctx, cudaFreeAsync(p, ctx->stream));
  m.owned.clear();
  return CAS_OK;
}

// Device memory a stream-ordered allocation can still get: the device's free
// memory plus what the pool holds reserved but unused (freed allocations it
// keeps, since its release threshold is unbounded).  cudaMemGetInfo alone
// would count the pool's idle reserve as taken, so sizes chosen from it would
// shrink after every large product.
double free_device_bytes(cas_ctx* ctx) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return 0.0;
  }
  double idle = 0.0;
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;  // 64-bit attribute values
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
    idle = (double)(reserved - used);
  cudaGetLastError();
  return (double)free_b + idle;
}

cas_status dev_alloc(cas_ctx* ctx, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, e == cudaErrorMemoryAllocation ? CAS_ERR_OOM : CAS_ERR_CUDA,
                   "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  return CAS_OK;
}

// Host memory for C: 2 MiB-aligned and marked for transparent huge pages,
// so first touch faults once per 2 MiB instead of once per 4 KiB (the copy
// into fresh 4 KiB pages runs at a third of the DMA rate).  Freed with free().
void* host_alloc_huge(size_t bytes) {
  constexpr size_t kHuge = size_t(2) << 20;
  const size_t len = (bytes + kHuge - 1) / kHuge * kHuge;
  void* p = nullptr;
  if (posix_memalign(&p, kHuge, len ? len : kHuge) != 0) return nullptr;
  madvise(p, len ? len : kHuge, MADV_HUGEPAGE);  // advisory: ignored where THP is off
  return p;
}

// Host blocks for returned C arrays.  A block released through cas_csr_free
// stays with the context, its pages resident, and serves the next output of
// up to its size (but not one under half of it); a context keeps at most
// kHostCacheShare of physical memory this way and frees the rest.  Fresh
// pages cost a fault per 2 MiB during the copy; resident ones let the copy
// run at the DMA rate.
constexpr double kHostCacheShare = 0.6;

// Every cached block of every context is recorded in one process-wide map
// from the block to the context that allocated it, and all host-block
// bookkeeping (the map, and each context's host_blocks, host_free and
// host_pinned) is changed under one mutex.  So a block can be returned through
// any context, or none: cas_csr_free(NULL, C) or a call with another context
// finds the owner, unregisters the block from CUDA if the owner had
// registered it, and removes it from the owner's records before freeing it.
std::mutex g_host_mu;
std::unordered_map<void*, cas_ctx*> g_host_owner;

void* host_take(cas_ctx* ctx, size_t bytes) {
  std::lock_guard<std::mutex> lock(g_host_mu);
  size_t best = SIZE_MAX;
  size_t bi = 0;
  for (size_t i = 0; i < ctx->host_free.size(); ++i) {
    const size_t cap = ctx->host_free[i].second;
    if (cap >= bytes && cap / 2 <= bytes && cap < best) {
      best = cap;
      bi = i;
    }
  }
  if (best != SIZE_MAX) {
    void* p = ctx->host_free[bi].first;
    ctx->host_free_bytes -= best;
    ctx->host_free.erase(ctx->host_free.begin() + (std::ptrdiff_t)bi);
    return p;
  }
  void* p = host_alloc_huge(bytes);
  if (p) {
    ctx->host_blocks[p] = bytes;
    g_host_owner[p] = ctx;
  }
  return p;
}

// A block the cache keeps (at least kPinMin bytes) is registered with CUDA
// when it enters the cache, once: a later output in it is copied from the
// device by DMA directly, without the staging buffers.  The cost of
// registering falls on the cas_csr_free that returns the block.
// Registered memory cannot be paged out, so all contexts of the process
// together register at most kPinShare of physical memory; past that, blocks
// stay unregistered and their outputs go through staging.
constexpr size_t kPinMin = size_t(64) << 20;
constexpr double kPinShare = 0.6;
std::atomic<size_t> g_pinned_bytes{0};

size_t pin_length(size_t bytes) {
  constexpr size_t kHuge = size_t(2) << 20;  // the allocation's length, as host_alloc_huge rounds it
  return (bytes + kHuge - 1) / kHuge * kHuge;
}

void host_pin(cas_ctx* ctx, void* p, size_t bytes) {
  if (ctx->host_pin_off || bytes < kPinMin || ctx->host_pinned.count(p)) return;
  static const double phys = (double)sysconf(_SC_PHYS_PAGES) * (double)sysconf(_SC_PAGESIZE);
  const size_t len = pin_length(bytes);
  if ((double)(g_pinned_bytes.fetch_add(len) + len) > kPinShare * phys) {
    g_pinned_bytes.fetch_sub(len);
    return;
  }
  if (cudaHostRegister(p, len, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    g_pinned_bytes.fetch_sub(len);
    ctx->host_pin_off = true;
    return;
  }
  ctx->host_pinned.insert(p);
}

void host_unpin(cas_ctx* ctx, void* p, size_t bytes) {
  if (ctx->host_pinned.erase(p)) {
    cudaHostUnregister(p);
    g_pinned_bytes.fetch_sub(pin_length(bytes));
  }
}

// Returns a host block of a C.  A block of ctx's own cache goes back to it
// (or is freed when the cache is full); a block of another context is
// released from that context's records and freed; any other pointer is freed.
void host_give(cas_ctx* ctx, void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_host_mu);
  auto own = g_host_owner.find(p);
  if (own == g_host_owner.end()) {
    free(p);
    return;
  }
  cas_ctx* owner = own->second;
  auto it = owner->host_blocks.find(p);
  static const double phys = (double)sysconf(_SC_PHYS_PAGES) * (double)sysconf(_SC_PAGESIZE);
  if (owner != ctx || (double)(owner->host_free_bytes + it->second) > kHostCacheShare * phys) {
    host_unpin(owner, p, it->second);
    owner->host_blocks.erase(it);
    g_host_owner.erase(own);
    free(p);
    return;
  }
  host_pin(ctx, p, it->second);
  ctx->host_free.emplace_back(p, it->second);
  ctx->host_free_bytes += it->second;
}

// Copies out of a staging buffer with non-temporal stores: the destination
// lines are written without being read first, which is a third less memory
// traffic than a plain copy of data that is not reused soon.  Falls back to
// memcpy for a misaligned destination and for the tail.
__attribute__((target("avx2"))) void stream_copy(char* d, const char* s, size_t n) {
  if ((reinterpret_cast<uintptr_t>(d) & 31) || (reinterpret_cast<uintptr_t>(s) & 31)) {
    memcpy(d, s, n);
    return;
  }
  const size_t v = n / 128;
  for (size_t i = 0; i < v; ++i) {
    const __m256i* src = reinterpret_cast<const __m256i*>(s) + 4 * i;
    __m256i* dst = reinterpret_cast<__m256i*>(d) + 4 * i;
    const __m256i a = _mm256_load_si256(src), b = _mm256_load_si256(src + 1);
    const __m256i c = _mm256_load_si256(src + 2), e = _mm256_load_si256(src + 3);
    _mm256_stream_si256(dst, a);
    _mm256_stream_si256(dst + 1, b);
    _mm256_stream_si256(dst + 2, c);
    _mm256_stream_si256(dst + 3, e);
  }
  memcpy(d + v * 128, s + v * 128, n - v * 128);
  _mm_sfence();
}

// int32 -> int64 widening copy with non-temporal stores (n int32 values).
__attribute__((target("avx2"))) void stream_widen(int64_t* d, const int32_t* s, size_t n) {
  size_t i = 0;
  if (!(reinterpret_cast<uintptr_t>(d) & 31) && !(reinterpret_cast<uintptr_t>(s) & 15)) {
    for (; i + 8 <= n; i += 8) {
      const __m128i lo = _mm_load_si128(reinterpret_cast<const __m128i*>(s + i));
      const __m128i hi = _mm_load_si128(reinterpret_cast<const __m128i*>(s + i + 4));
      _mm256_stream_si256(reinterpret_cast<__m256i*>(d + i), _mm256_cvtepi32_epi64(lo));
      _mm256_stream_si256(reinterpret_cast<__m256i*>(d + i + 4), _mm256_cvtepi32_epi64(hi));
    }
    _mm_sfence();
  }
  for (; i < n; ++i) d[i] = s[i];
}

// Device -> pageable host copy through pinned staging buffers: the DMA of
// chunk i runs while host threads move chunk i-1 out of staging.  With
// `widen`, the source holds int32 and the destination int64 (bytes counts
// the source).
constexpr int kStageBufs = 3;
cas_status d2h_staged(cas_ctx* ctx, void* dst, const void* src, size_t bytes, bool widen = false) {
  if (bytes == 0) return CAS_OK;
  if (!ctx->h_stage[0]) {
    for (int i = 0; i < kStageBufs; ++i) {
      CAS_CUDA(ctx, cudaMallocHost(&ctx->h_stage[i], kStageBytes));
      CAS_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_stage[i], cudaEventDisableTiming));
    }
  }
  const size_t nchunk = (bytes + kStageBytes - 1) / kStageBytes;
  auto issue = [&](size_t i) -> cas_status {
    const size_t off = i * kStageBytes, len = std::min(kStageBytes, bytes - off);
    CAS_CUDA(ctx, cudaMemcpyAsync(ctx->h_stage[i % kStageBufs], static_cast<const char*>(src) + off, len,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CAS_CUDA(ctx, cudaEventRecord(ctx->ev_stage[i % kStageBufs], ctx->stream));
    return CAS_OK;
  };
  for (size_t i = 0; i < std::min<size_t>(kStageBufs - 1, nchunk); ++i) CAS_TRY(issue(i));
  for (size_t j = 0; j < nchunk; ++j) {
    if (j + kStageBufs - 1 < nchunk) CAS_TRY(issue(j + kStageBufs - 1));
    const size_t off = j * kStageBytes, len = std::min(kStageBytes, bytes - off);
    CAS_CUDA(ctx, cudaEventSynchronize(ctx->ev_stage[j % kStageBufs]));
    const char* s = static_cast<const char*>(ctx->h_stage[j % kStageBufs]);
    const int64_t pieces = (int64_t)((len + (1 << 20) - 1) >> 20);
    if (widen) {
      const int32_t* s32 = reinterpret_cast<const int32_t*>(s);
      int64_t* d64 = static_cast<int64_t*>(dst) + off / 4;
#pragma omp parallel for schedule(static)
      for (int64_t p = 0; p < pieces; ++p) {
        const size_t o = (size_t)p << 18, e = std::min(o + ((size_t)1 << 18), len / 4);
        stream_widen(d64 + o, s32 + o, e - o);
      }
    } else {
      char* d = static_cast<char*>(dst) + off;
#pragma omp parallel for schedule(static)
      for (int64_t p = 0; p < pieces; ++p) {
        const size_t o = (size_t)p << 20;
        stream_copy(d + o, s + o, std::min((size_t)1 << 20, len - o));
      }
    }
  }
  return CAS_OK;
}

// Device -> host copy of one output array: by DMA straight into a block the
// context has registered, else through the staging buffers.
bool host_is_pinned(cas_ctx* ctx, void* p) {
  std::lock_guard<std::mutex> lock(g_host_mu);
  return ctx->host_pinned.count(p) != 0;
}

cas_status d2h_out(cas_ctx* ctx, void* dst, const void* src, size_t bytes, bool widen = false) {
  if (bytes > 0 && !widen && host_is_pinned(ctx, dst)) {
    CAS_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h_direct += (double)bytes;
    return CAS_OK;
  }
  return d2h_staged(ctx, dst, src, bytes, widen);
}

cas_status basic_checks(cas_ctx* ctx, const cas_csr* M, const char* name) {
  if (!M) return set_err(ctx, CAS_ERR_BAD_INPUT, "%s is NULL", name);
  if (M->num_row < 0 || M->num_col < 0 || M->num_nnz < 0 || M->num_row > INT32_MAX || M->num_col > INT32_MAX)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "%s has an invalid shape", name);
  if (!M->row_ptrs || (M->num_nnz > 0 && (!M->cols || !M->rats)))
    return set_err(ctx, CAS_ERR_BAD_INPUT, "%s has NULL arrays", name);
  if (M->val_type != CAS_VAL_F64 && M->val_type != CAS_VAL_I32)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "%s has an unknown value type", name);
  if (M->on_device ? M->col_bytes != 4 : (M->col_bytes != 4 && M->col_bytes != 8))
    return set_err(ctx, CAS_ERR_BAD_INPUT, "%s has column width %d", name, M->col_bytes);
  return CAS_OK;
}

cas_status to_device(cas_ctx* ctx, const cas_csr* M, DevMat& out, double& h2d) {
  out.csr.nrow = M->num_row;
  out.csr.ncol = M->num_col;
  out.nnz = M->num_nnz;
  out.vt = M->val_type;
  const size_t vbytes = M->val_type == CAS_VAL_F64 ? 8 : 4;
  if (M->on_device) {
    out.csr.rp = M->row_ptrs;
    out.csr.col = static_cast<const int32_t*>(M->cols);
    out.csr.val = M->rats;
    return CAS_OK;
  }
  if (M->row_ptrs[0] != 0 || M->row_ptrs[M->num_row] != M->num_nnz)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "row pointers do not span [0, num_nnz]");
  void *rp, *col, *val;
  CAS_TRY(dev_alloc(ctx, &rp, sizeof(int64_t) * (M->num_row + 1)));
  out.owned.push_back(rp);
  CAS_TRY(dev_alloc(ctx, &col, sizeof(int32_t) * M->num_nnz));
  out.owned.push_back(col);
  CAS_TRY(dev_alloc(ctx, &val, vbytes * M->num_nnz));
  out.owned.push_back(val);
  CAS_CUDA(ctx, cudaMemcpyAsync(rp, M->row_ptrs, sizeof(int64_t) * (M->num_row + 1), cudaMemcpyHostToDevice, ctx->stream));
  if (M->col_bytes == 4) {
    CAS_CUDA(ctx, cudaMemcpyAsync(col, M->cols, sizeof(int32_t) * M->num_nnz, cudaMemcpyHostToDevice, ctx->stream));
    h2d += sizeof(int32_t) * (double)M->num_nnz;
  } else {
    // the reference's int64 columns: narrowed on the host
    std::vector<int32_t> tmp((size_t)M->num_nnz);
    const int64_t* c64 = static_cast<const int64_t*>(M->cols);
    for (int64_t i = 0; i < M->num_nnz; ++i) {
      if (c64[i] < 0 || c64[i] > INT32_MAX) return set_err(ctx, CAS_ERR_BAD_INPUT, "column index out of int32 range");
      tmp[(size_t)i] = (int32_t)c64[i];
    }
    CAS_CUDA(ctx, cudaMemcpyAsync(col, tmp.data(), sizeof(int32_t) * M->num_nnz, cudaMemcpyHostToDevice, ctx->stream));
    CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    h2d += sizeof(int64_t) * (double)M->num_nnz;
  }
  CAS_CUDA(ctx, cudaMemcpyAsync(val, M->rats, vbytes * M->num_nnz, cudaMemcpyHostToDevice, ctx->stream));
  h2d += sizeof(int64_t) * (double)(M->num_row + 1) + vbytes * (double)M->num_nnz;
  out.csr.rp = static_cast<const int64_t*>(rp);
  out.csr.col = static_cast<const int32_t*>(col);
  out.csr.val = val;
  return CAS_OK;
}

}  // namespace

// ============================================================ input check
namespace cas {
// One warp per row: row pointers non-decreasing and within [0, nnz], column
// indices in [0, ncol); flags[1] is set when some row is not sorted.
__global__ void k_check_csr(Csr M, int64_t nnz, unsigned long long* flags) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < M.nrow; r += nw) {
    const int64_t s = M.rp[r], e = M.rp[r + 1];
    if (s < 0 || e < s || e > nnz) {
      if (lane == 0) atomicOr(&flags[0], 1ull);
      continue;
    }
    bool bad = false, unsorted = false;
    for (int64_t j = s + lane; j < e; j += 32) {
      const int32_t c = M.col[j];
      bad |= (uint64_t)c >= (uint64_t)M.ncol;
      if (j + 1 < e) unsorted |= M.col[j + 1] < c;
    }
    if (__any_sync(kFull, bad) && lane == 0) atomicOr(&flags[0], 1ull);
    if (__any_sync(kFull, unsorted) && lane == 0) atomicOr(&flags[1], 1ull);
  }
}
}  // namespace cas

namespace {

struct Call {
  DevMat A, B;
  int64_t m = 0, ncol = 0;
  int vt = CAS_VAL_F64;
  int64_t* row_flp = nullptr;
  int64_t* row_nz = nullptr;
  int32_t* rows = nullptr;
  int32_t* ovf = nullptr;  // rows the bucketed ESC kernel hands to the radix-sort ESC kernel
  int64_t* partial = nullptr;
  int64_t nparts = 0;
  bool b_sorted = true;
  bool ovf_launched = false;
  int64_t symb_count[cas::kSymbBins] = {};
  int64_t numc_count[cas::kNumcBins] = {};
  int64_t flop = 0, max_flp = 0;
  // fused rows (cas_spgemm with ESC or hybrid accumulation)
  int fuse = 0;
  int64_t nf = 0, f_flop = 0, f_bound = 0, f_nnza = 0;
  int32_t* frows = nullptr;
  int64_t* fpos = nullptr;
  unsigned long long* fstatus = nullptr;
  bool ovf_preset = false;
  // bitmaps of heavy rows kept by the symbolic kernel for the numeric one
  uint32_t* dbits = nullptr;
  int32_t* dslot = nullptr;
  int saved_slices = 1;  // bitmap slots kept per row in dbits
  // the symbolic phase's split rows: their slice bitmaps, and each row's slot
  // in them (-1 for other rows); kept for the numeric setup of split rows
  uint32_t* hbits = nullptr;
  int32_t* hslot = nullptr;
  std::vector<void*> heavy_tmp;  // the rest of the symbolic split's scratch
};

cas_status fork(cas_ctx* ctx) {
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
  for (int i = 0; i < kAux; ++i) CAS_CUDA(ctx, cudaStreamWaitEvent(ctx->aux[i], ctx->ev_fork, 0));
  return CAS_OK;
}
cas_status join(cas_ctx* ctx) {
  for (int i = 0; i < kAux; ++i) {
    CAS_CUDA(ctx, cudaEventRecord(ctx->ev_join[i], ctx->aux[i]));
    CAS_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join[i], 0));
  }
  return CAS_OK;
}

cas_status scratch_alloc(cas_ctx* ctx, Call& c) {
  CAS_TRY(dev_alloc(ctx, (void**)&c.row_flp, sizeof(int64_t) * (c.m + 1)));
  CAS_TRY(dev_alloc(ctx, (void**)&c.row_nz, sizeof(int64_t) * (c.m + 1)));
  CAS_TRY(dev_alloc(ctx, (void**)&c.rows, sizeof(int32_t) * (c.m + 1)));
  CAS_TRY(dev_alloc(ctx, (void**)&c.ovf, sizeof(int32_t) * (c.m + 1)));
  c.nparts = (c.m + 1 + cas::kScanTile - 1) / cas::kScanTile;
  CAS_TRY(dev_alloc(ctx, (void**)&c.partial, sizeof(int64_t) * (c.nparts + 1)));
  return CAS_OK;
}

cas_status scratch_free(cas_ctx* ctx, Call& c) {
  void* ps[] = {c.row_flp, c.row_nz, c.rows, c.ovf, c.partial, c.frows, c.fpos, c.fstatus, c.dbits, c.dslot};
  for (void* p : ps)
    if (p) CAS_CUDA(ctx, cudaFreeAsync(p, ctx->stream));
  c.row_flp = c.row_nz = nullptr;
  c.rows = c.ovf = nullptr;
  c.partial = nullptr;
  c.frows = nullptr;
  c.fpos = nullptr;
  c.fstatus = nullptr;
  c.dbits = nullptr;
  c.dslot = nullptr;
  for (void* p : c.heavy_tmp) CAS_CUDA(ctx, cudaFreeAsync(p, ctx->stream));
  c.heavy_tmp.clear();
  c.hbits = nullptr;
  c.hslot = nullptr;
  return CAS_OK;
}

// exclusive scan of in[0..n-1) into out[0..n), total of in into counter slot
cas_status launch_scan(cas_ctx* ctx, int64_t* out, const int64_t* in, int64_t n, int64_t* partial,
                       int64_t* total_out) {
  using namespace cas;
  if (n <= 0) return CAS_OK;
  const int64_t n_in = n - 1;
  const int64_t nparts = (n + kScanTile - 1) / kScanTile;
  k_scan_partials<<<(unsigned)nparts, kScanBlock, 0, ctx->stream>>>(in, n_in, partial);
  CAS_TRY(check_launch(ctx, "k_scan_partials"));
  k_scan_top<<<1, kScanBlock, 0, ctx->stream>>>(partial, nparts, total_out);
  CAS_TRY(check_launch(ctx, "k_scan_top"));
  k_scan_apply<<<(unsigned)nparts, kScanBlock, 0, ctx->stream>>>(in, n_in, partial, out, n);
  CAS_TRY(check_launch(ctx, "k_scan_apply"));
  return CAS_OK;
}

// ------------------------------------------------------------------ INIT
// Row pointers and column indices of A and B in range (an error if not), and
// whether B's rows are sorted by column (c.b_sorted).  Synchronises.
cas_status check_inputs(cas_ctx* ctx, Call& c) {
  using namespace cas;
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotCheck, 0, sizeof(unsigned long long) * 4, ctx->stream));
  const int g = grid_for(std::max<int64_t>(c.A.csr.nrow, c.B.csr.nrow) * 32, 256, ctx->sm_count * 16);
  Csr a = c.A.csr;
  a.ncol = c.B.csr.nrow;  // A's columns index B's rows
  k_check_csr<<<g, 256, 0, ctx->stream>>>(a, c.A.nnz, ctx->d_counts + kSlotCheck);
  CAS_TRY(check_launch(ctx, "k_check_csr"));
  k_check_csr<<<g, 256, 0, ctx->stream>>>(c.B.csr, c.B.nnz, ctx->d_counts + kSlotCheck + 2);
  CAS_TRY(check_launch(ctx, "k_check_csr"));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotCheck, ctx->d_counts + kSlotCheck, 4, ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->h_counts[kSlotCheck] || ctx->h_counts[kSlotCheck + 2])
    return set_err(ctx, CAS_ERR_BAD_INPUT, "invalid CSR input: row pointers or column indices out of range");
  c.b_sorted = ctx->h_counts[kSlotCheck + 3] == 0;
  return CAS_OK;
}

// With `validate`, checks the inputs first (check_inputs); without, c.b_sorted
// is the caller's (a row block of a checked product).
cas_status phase_init(cas_ctx* ctx, Call& c, bool validate) {
  using namespace cas;
  if (validate) CAS_TRY(check_inputs(ctx, c));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts, 0, sizeof(unsigned long long) * kCountSlots, ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(DevStatus), ctx->stream));
  CAS_TRY(scratch_alloc(ctx, c));
  if (c.m > 0) {
    k_flp<256><<<grid_for(c.m * 32, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        c.A.csr, c.B.csr, c.ncol, c.row_flp, ctx->d_counts + kSlotTotals, ctx->d_counts + kSlotSymb, ctx->d_status,
        c.fuse, ctx->d_counts + kSlotFused);
    CAS_TRY(check_launch(ctx, "k_flp"));
  }
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev, ctx->d_counts, kCountSlots, ctx->stream));
  CAS_TRY(check_status(ctx));  // synchronises
  c.flop = (int64_t)ctx->h_counts[kSlotTotals];
  c.max_flp = (int64_t)ctx->h_counts[kSlotTotals + 1];
  c.nf = (int64_t)ctx->h_counts[kSlotFused];
  c.f_flop = (int64_t)ctx->h_counts[kSlotFused + 1];
  c.f_bound = (int64_t)ctx->h_counts[kSlotFused + 2];
  c.f_nnza = (int64_t)ctx->h_counts[kSlotFused + 3];
  unsigned long long* cur = ctx->h_counts + kSlotCursor;
  unsigned long long off = 0;
  for (int b = 0; b < kSymbBins; ++b) {
    c.symb_count[b] = (int64_t)ctx->h_counts[kSlotSymb + b];
    cur[b] = off;
    off += ctx->h_counts[kSlotSymb + b];
  }
  if (c.m > 0) {
    CAS_CUDA(ctx, cudaMemcpyAsync(ctx->d_counts + kSlotCursor, cur, sizeof(unsigned long long) * kSymbBins,
                                  cudaMemcpyHostToDevice, ctx->stream));
    k_bin_scatter_symb<<<grid_for(c.m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        c.m, c.row_flp, c.ncol, ctx->d_counts + kSlotCursor, c.rows, c.fuse);
    CAS_TRY(check_launch(ctx, "k_bin_scatter_symb"));
  }
  if (c.nf > 0) {
    // the fused rows in ascending order: marks (in row_nz, cleared before the
    // symbolic kernels), their scan, the scatter
    CAS_TRY(dev_alloc(ctx, (void**)&c.fpos, sizeof(int64_t) * (c.m + 1)));
    CAS_TRY(dev_alloc(ctx, (void**)&c.frows, sizeof(int32_t) * c.nf));
    CAS_TRY(dev_alloc(ctx, (void**)&c.fstatus, sizeof(unsigned long long) * c.nf));
    const int g = grid_for(c.m, 256, ctx->sm_count * 8);
    k_fused_mark<<<g, 256, 0, ctx->stream>>>(c.m, c.row_flp, c.fuse, c.row_nz);
    CAS_TRY(check_launch(ctx, "k_fused_mark"));
    CAS_TRY(launch_scan(ctx, c.fpos, c.row_nz, c.m + 1, c.partial, nullptr));
    k_fused_scatter<<<g, 256, 0, ctx->stream>>>(c.m, c.row_flp, c.fuse, c.fpos, c.frows);
    CAS_TRY(check_launch(ctx, "k_fused_scatter"));
  }
  return CAS_OK;
}

// ------------------------------------------------------------- FUSED ROWS
// The fused ESC kernel over the fused rows, in row order: each writes its row
// of C at known[r] (the scan of the other rows' counts) plus the counts of the
// fused rows before it, and its count into row_nz.
template <typename VIn>
cas_status launch_fused(cas_ctx* ctx, Call& c, const int64_t* known, int32_t* ccol, void* cval, int64_t cap) {
  using namespace cas;
  using AT = typename Acc<VIn>::T;
  if (c.nf == 0) return CAS_OK;
  unsigned int* ovf_count = reinterpret_cast<unsigned int*>(ctx->d_counts + kSlotOvf);
  CAS_CUDA(ctx, cudaMemsetAsync(ovf_count, 0, sizeof(unsigned int), ctx->stream));
  c.ovf_preset = true;
  CAS_CUDA(ctx, cudaMemsetAsync(c.fstatus, 0, sizeof(unsigned long long) * c.nf, ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotFused + 4, 0, sizeof(unsigned long long), ctx->stream));
  Fused fu{c.frows, ctx->d_counts + kSlotFused + 4, c.fstatus, known, c.row_nz, cap};
  if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_fused[0], ctx->stream));
  if (ctx->esc_form == 1)
    k_numc_esc_idx<256, (int)kFusedHi, 11, VIn, true>
        <<<(unsigned)c.nf, 256, smem_numc_esc_idx<(int)kFusedHi, 11, VIn>(), ctx->stream>>>(
            nullptr, c.A.csr, c.B.csr, c.b_sorted ? 1 : 0, nullptr, ccol, static_cast<AT*>(cval), c.ovf, ovf_count,
            ctx->d_status, fu);
  else if (ctx->esc_form == 2)
    k_numc_esc_idx<256, (int)kFusedHi, 11, VIn, true, true>
        <<<(unsigned)c.nf, 256, smem_numc_esc_idx<(int)kFusedHi, 11, VIn>(), ctx->stream>>>(
            nullptr, c.A.csr, c.B.csr, c.b_sorted ? 1 : 0, nullptr, ccol, static_cast<AT*>(cval), c.ovf, ovf_count,
            ctx->d_status, fu);
  else
    k_numc_esc_msd<256, (int)kFusedHi, 11, VIn, true>
        <<<(unsigned)c.nf, 256, smem_numc_esc_msd<(int)kFusedHi, 11, VIn>(), ctx->stream>>>(
            nullptr, c.A.csr, c.B.csr, c.b_sorted ? 1 : 0, nullptr, ccol, static_cast<AT*>(cval), c.ovf, ovf_count,
            ctx->d_status, fu);
  CAS_TRY(check_launch(ctx, "k_numc_esc_msd (fused)"));
  if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_fused[1], ctx->stream));
  return CAS_OK;
}

constexpr int64_t kSplitScratch = int64_t(8) << 30;  // at most 8 GiB of slice bitmaps per phase

// The symbolic phase's split rows (see k_heavy_plan in cas_kernels.cu): the
// dense symbolic rows of at least kSplitProducts products, up to the scratch
// cap, get their slice bitmaps built by parts over many blocks and their
// counts from those bitmaps; the rest stay in `rows`, and their number in n.
cas_status symb_split_heavy(cas_ctx* ctx, Call& c, int32_t*& rows, int64_t& n, int64_t* row_nz, cudaStream_t s) {
  using namespace cas;
  const int64_t max_slices = (c.ncol + kRankCols - 1) / kRankCols;
  const int64_t cap = (int64_t)((double)kSplitScratch * ctx->mem_share) / (max_slices * (kRankCols / 8));
  auto alloc = [&](void** p, size_t bytes) -> cas_status {
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, e == cudaErrorMemoryAllocation ? CAS_ERR_OOM : CAS_ERR_CUDA,
                     "device allocation of %zu bytes for the split rows failed", bytes);
    }
    c.heavy_tmp.push_back(*p);
    return CAS_OK;
  };
  int32_t *heavy = nullptr, *light = nullptr;
  unsigned long long* counts = nullptr;
  CAS_TRY(alloc((void**)&c.hslot, sizeof(int32_t) * (size_t)(c.m + 1)));
  CAS_TRY(alloc((void**)&heavy, sizeof(int32_t) * (size_t)n));
  CAS_TRY(alloc((void**)&light, sizeof(int32_t) * (size_t)n));
  CAS_TRY(alloc((void**)&counts, 2 * sizeof(unsigned long long)));
  CAS_CUDA(ctx, cudaMemsetAsync(c.hslot, 0xFF, sizeof(int32_t) * (size_t)(c.m + 1), s));
  CAS_CUDA(ctx, cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s));
  k_split_dense_rows<<<grid_for(n, 256, ctx->sm_count * 4), 256, 0, s>>>(rows, n, c.row_flp, cap, heavy, light, counts,
                                                                          c.hslot);
  CAS_TRY(check_launch(ctx, "k_split_dense_rows"));
  CAS_TRY(fetch_words(ctx, ctx->h_misc_dev, counts, 2, s));
  CAS_CUDA(ctx, cudaStreamSynchronize(s));
  const unsigned long long h[2] = {ctx->h_misc[0], ctx->h_misc[1]};
  const int64_t nh = std::min<int64_t>((int64_t)h[0], cap);
  rows = light;
  n = (int64_t)h[1];
  if (nh == 0) return CAS_OK;
  HeavyPlan hp{};
  hp.rows = heavy;
  hp.n = nh;
  hp.max_slices = (int)max_slices;
  CAS_TRY(alloc((void**)&hp.bits, (size_t)nh * max_slices * (kRankCols / 8)));
  CAS_TRY(alloc((void**)&hp.slice_base, sizeof(int64_t) * (size_t)nh * max_slices));
  CAS_TRY(alloc((void**)&hp.lo, sizeof(int64_t) * (size_t)nh));
  CAS_TRY(alloc((void**)&hp.hi, sizeof(int64_t) * (size_t)nh));
  CAS_TRY(alloc((void**)&hp.nslices, sizeof(int32_t) * (size_t)nh));
  CAS_TRY(alloc((void**)&hp.products, sizeof(int64_t) * (size_t)nh));
  CAS_TRY(alloc((void**)&hp.nparts, sizeof(int64_t) * (size_t)nh));
  CAS_TRY(alloc((void**)&hp.parts, sizeof(int64_t) * (size_t)(nh + 1)));
  CAS_TRY(alloc((void**)&hp.apre, sizeof(int64_t) * (size_t)(c.A.nnz > 0 ? c.A.nnz : 1)));
  CAS_TRY(alloc((void**)&hp.ticket, sizeof(unsigned long long)));
  c.hbits = hp.bits;
  CAS_CUDA(ctx, cudaMemsetAsync(hp.ticket, 0, sizeof(unsigned long long), s));
  k_heavy_plan<512><<<(unsigned)nh, 512, 0, s>>>(hp, c.A.csr, c.B.csr, c.ncol, c.b_sorted ? 1 : 0, ctx->d_status);
  CAS_TRY(check_launch(ctx, "k_heavy_plan"));
  k_scan_one_block<<<1, 1024, 0, s>>>(hp.nparts, nh, hp.parts);
  CAS_TRY(check_launch(ctx, "k_scan_one_block"));
  int per_sm = 0;
  CAS_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_heavy_bits<512>, 512, smem_symb_dense<512>()));
  k_heavy_bits<512><<<std::max(1, per_sm) * ctx->sm_count, 512, smem_symb_dense<512>(), s>>>(hp, c.A.csr, c.B.csr,
                                                                                             ctx->d_status);
  CAS_TRY(check_launch(ctx, "k_heavy_bits"));
  k_heavy_count<512><<<(unsigned)nh, 512, 0, s>>>(hp, row_nz);
  CAS_TRY(check_launch(ctx, "k_heavy_count"));
  return CAS_OK;
}

// ------------------------------------------------------------------ SYMB
cas_status launch_symb_bins(cas_ctx* ctx, Call& c, int64_t* row_nz) {
  using namespace cas;
  CAS_CUDA(ctx, cudaMemsetAsync(row_nz, 0, sizeof(int64_t) * (c.m + 1), ctx->stream));
  CAS_TRY(fork(ctx));
  int64_t off[kSymbBins + 1] = {0};
  for (int b = 0; b < kSymbBins; ++b) off[b + 1] = off[b] + c.symb_count[b];
  // heaviest bins first, each on its own stream
  const int order[] = {kSB_Dense, kSB_H32K, kSB_H16K, kSB_H8K, kSB_H4K, kSB_H2K, kSB_H1K, kSB_Tiny};
  int si = 0;
  for (int b : order) {
    const int64_t n = c.symb_count[b];
    if (n == 0) continue;
    const int32_t* rows = c.rows + off[b];
    cudaStream_t s = ctx->profile ? ctx->stream : ctx->aux[si++ % kAux];  // profiling: one bin at a time
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_symb[0][b], s));
    switch (b) {
      case kSB_Tiny:
        k_symb_tiny<256><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(rows, n, c.A.csr, c.B.csr, row_nz, ctx->d_status);
        break;
#define CAS_SYMB_CASE(bin, BLK, TB, SEG)                                                              \
      case bin:                                                                                     \
        k_symb_hash<BLK, TB, SEG><<<(unsigned)n, BLK, smem_symb_hash<BLK, TB, SEG>(), s>>>(          \
            rows, c.A.csr, c.B.csr, row_nz, ctx->d_status);                                         \
        break;
      CAS_SYMB_SHAPES(CAS_SYMB_CASE)
#undef CAS_SYMB_CASE
      case kSB_Dense: {
        if (!c.b_sorted && c.ncol > kDenseChunkBits)
          return set_err(ctx, CAS_ERR_BAD_INPUT, "heavy rows over more than %d columns need B rows sorted by column", kDenseChunkBits);
        int32_t* drows = const_cast<int32_t*>(rows);
        int64_t nd = n;
        if (ctx->heavy_split) {
          CAS_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
          CAS_CUDA(ctx, cudaStreamWaitEvent(s, ctx->ev_fork, 0));
          CAS_TRY(symb_split_heavy(ctx, c, drows, nd, row_nz, s));
        }
        if (nd == 0) break;
        // bitmaps kept for the numeric kernel: every slice of each row when that fits a quarter
        // of the free device memory, at most 24 GiB (and at least kSavedBitmapBytes), else
        // one-slice rows only
        const double free_b = free_device_bytes(ctx);
        const double cap = ctx->mem_share * std::max(kSavedBitmapBytes, std::min(24.0 * (1ull << 30), 0.25 * free_b));
        const int64_t max_slices = (c.ncol + kRankCols - 1) / kRankCols;
        c.saved_slices = (double)nd * max_slices * (kRankCols / 8) <= cap ? (int)max_slices : 1;
        if ((double)nd * c.saved_slices * (kRankCols / 8) <= cap) {
          CAS_TRY(dev_alloc(ctx, (void**)&c.dbits, (size_t)nd * c.saved_slices * (kRankCols / 8)));
          CAS_TRY(dev_alloc(ctx, (void**)&c.dslot, sizeof(int32_t) * (c.m + 1)));
          CAS_CUDA(ctx, cudaMemsetAsync(c.dslot, 0xFF, sizeof(int32_t) * (c.m + 1), ctx->stream));
          CAS_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
          CAS_CUDA(ctx, cudaStreamWaitEvent(s, ctx->ev_fork, 0));
        }
        k_symb_dense<512><<<(unsigned)nd, 512, smem_symb_dense<512>(), s>>>(drows, c.A.csr, c.B.csr, c.ncol,
                                                                             c.b_sorted ? 1 : 0, row_nz, c.dbits,
                                                                             c.dslot, c.saved_slices, ctx->d_status);
        break;
      }
    }
    CAS_TRY(check_launch(ctx, "symbolic bin"));
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_symb[1][b], s));
  }
  CAS_TRY(join(ctx));
  return CAS_OK;
}

// ------------------------------------------------------------------ MGMT
cas_status numc_bins(cas_ctx* ctx, Call& c, const int64_t* crp, int mode) {
  using namespace cas;
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotNumc, 0, sizeof(unsigned long long) * kNumcBins, ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotBinSums, 0, sizeof(unsigned long long) * 3 * kNumcBins,
                                ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + kSlotHeavy, 0, sizeof(unsigned long long) * kHeavyClasses,
                                ctx->stream));
  if (c.m > 0) {
    k_bin_count_numc<<<grid_for(c.m, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(
        c.m, c.row_flp, crp, c.A.csr.rp, mode, ctx->acc_thres, ctx->esc_max, ctx->hash_max,
        ctx->d_counts + kSlotNumc, ctx->d_counts + kSlotBinSums, ctx->d_counts + kSlotHeavy);
    CAS_TRY(check_launch(ctx, "k_bin_count_numc"));
  }
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotNumc, ctx->d_counts + kSlotNumc, kNumcBins, ctx->stream));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotBinSums, ctx->d_counts + kSlotBinSums, 3 * kNumcBins, ctx->stream));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotHeavy, ctx->d_counts + kSlotHeavy, kHeavyClasses, ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long* cur = ctx->h_counts + kSlotCursor;
  unsigned long long off = 0;
  for (int b = 0; b < kNumcBins; ++b) {
    c.numc_count[b] = (int64_t)ctx->h_counts[kSlotNumc + b];
    cur[b] = off;
    if (b == kNB_Dense) {  // heaviest size class first
      unsigned long long* hc = ctx->h_counts + kSlotHeavyCur;
      unsigned long long o = off;
      for (int k = 0; k < kHeavyClasses; ++k) {
        hc[k] = o;
        o += ctx->h_counts[kSlotHeavy + k];
      }
    }
    off += ctx->h_counts[kSlotNumc + b];
  }
  if (c.m > 0) {
    CAS_CUDA(ctx, cudaMemcpyAsync(ctx->d_counts + kSlotCursor, cur, sizeof(unsigned long long) * kNumcBins,
                                  cudaMemcpyHostToDevice, ctx->stream));
    CAS_CUDA(ctx, cudaMemcpyAsync(ctx->d_counts + kSlotHeavyCur, ctx->h_counts + kSlotHeavyCur,
                                  sizeof(unsigned long long) * kHeavyClasses, cudaMemcpyHostToDevice, ctx->stream));
    k_bin_scatter_numc<<<grid_for(c.m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        c.m, c.row_flp, crp, mode, ctx->acc_thres, ctx->esc_max, ctx->hash_max, ctx->d_counts + kSlotCursor,
        ctx->d_counts + kSlotHeavyCur, c.rows);
    CAS_TRY(check_launch(ctx, "k_bin_scatter_numc"));
  }
  return CAS_OK;
}

// ------------------------------------------------------------------ NUMC
// One bucketed ESC bin: the index form for bins of more than 4096 products
// when esc_form is 1, else the column-and-value form.
template <int CAP, int NBB, typename VIn>
void launch_esc_bin(int esc_form, int64_t n, cudaStream_t s, const int32_t* rows, const cas::Csr& A, const cas::Csr& B,
                    int32_t b_sorted, const int64_t* crp, int32_t* ccol, typename cas::Acc<VIn>::T* cval, int32_t* ovf,
                    unsigned int* ovf_count, cas::DevStatus* st) {
  using namespace cas;
  if constexpr (CAP > 4096 && CAP <= 6144) {
    if (esc_form == 2) {
      k_numc_esc_idx<256, CAP, NBB, VIn, false, true><<<(unsigned)n, 256, smem_numc_esc_idx<CAP, NBB, VIn>(), s>>>(
          rows, A, B, b_sorted, crp, ccol, cval, ovf, ovf_count, st, Fused{});
      return;
    }
  }
  if constexpr (CAP > 4096) {
    if (esc_form >= 1) {
      k_numc_esc_idx<256, CAP, NBB, VIn><<<(unsigned)n, 256, smem_numc_esc_idx<CAP, NBB, VIn>(), s>>>(
          rows, A, B, b_sorted, crp, ccol, cval, ovf, ovf_count, st, Fused{});
      return;
    }
  }
  k_numc_esc_msd<256, CAP, NBB, VIn><<<(unsigned)n, 256, smem_numc_esc_msd<CAP, NBB, VIn>(), s>>>(
      rows, A, B, b_sorted, crp, ccol, cval, ovf, ovf_count, st, Fused{});
}

// The heaviest dense rows over several blocks (k_dense_setup, then
// k_dense_acc; see cas_kernels.cu), on stream s, with scratch allocated and
// freed on s: the slice bitmaps (64 KiB per row and slice), the per-row
// plan and the product prefix of every A entry.

template <typename VIn>
cas_status launch_heavy_split(cas_ctx* ctx, Call& c, const int32_t* rows, int64_t n, const int64_t* crp, int32_t* ccol,
                              typename cas::Acc<VIn>::T* cval, cudaStream_t s) {
  using namespace cas;
  HeavyPlan hp{};
  hp.rows = rows;
  hp.n = n;
  hp.max_slices = (int)((c.ncol + kRankCols - 1) / kRankCols);
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) -> cas_status {
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, e == cudaErrorMemoryAllocation ? CAS_ERR_OOM : CAS_ERR_CUDA,
                     "device allocation of %zu bytes for the split rows failed", bytes);
    }
    tmp.push_back(*p);
    return CAS_OK;
  };
  cas_status rc = [&]() -> cas_status {
    CAS_TRY(alloc((void**)&hp.bits, (size_t)n * hp.max_slices * (kRankCols / 8)));
    CAS_TRY(alloc((void**)&hp.slice_base, sizeof(int64_t) * (size_t)n * hp.max_slices));
    CAS_TRY(alloc((void**)&hp.lo, sizeof(int64_t) * (size_t)n));
    CAS_TRY(alloc((void**)&hp.hi, sizeof(int64_t) * (size_t)n));
    CAS_TRY(alloc((void**)&hp.nslices, sizeof(int32_t) * (size_t)n));
    CAS_TRY(alloc((void**)&hp.products, sizeof(int64_t) * (size_t)n));
    CAS_TRY(alloc((void**)&hp.nparts, sizeof(int64_t) * (size_t)n));
    CAS_TRY(alloc((void**)&hp.parts, sizeof(int64_t) * (size_t)(n + 1)));
    CAS_TRY(alloc((void**)&hp.apre, sizeof(int64_t) * (size_t)(c.A.nnz > 0 ? c.A.nnz : 1)));
    CAS_TRY(alloc((void**)&hp.ticket, sizeof(unsigned long long)));
    CAS_CUDA(ctx, cudaMemsetAsync(hp.ticket, 0, sizeof(unsigned long long), s));
    k_dense_setup<512, VIn><<<(unsigned)n, 512, smem_numc_dense<512, VIn>(), s>>>(
        hp, c.A.csr, c.B.csr, c.ncol, c.b_sorted ? 1 : 0, crp, ccol, cval, c.dbits, c.dslot, c.saved_slices, c.hbits,
        c.hslot, ctx->d_status);
    CAS_TRY(check_launch(ctx, "k_dense_setup"));
    k_scan_one_block<<<1, 1024, 0, s>>>(hp.nparts, n, hp.parts);
    CAS_TRY(check_launch(ctx, "k_scan_one_block"));
    int per_sm = 0;
    CAS_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dense_acc<512, VIn>, 512,
                                                                smem_numc_dense<512, VIn>()));
    const int grid = std::max(1, per_sm) * ctx->sm_count;
    k_dense_acc<512, VIn><<<grid, 512, smem_numc_dense<512, VIn>(), s>>>(hp, c.A.csr, c.B.csr, crp, cval,
                                                                       ctx->d_status);
    CAS_TRY(check_launch(ctx, "k_dense_acc"));
    return CAS_OK;
  }();
  for (void* p : tmp) cudaFreeAsync(p, s);
  return rc;
}

template <typename VIn>
cas_status launch_numc_bins(cas_ctx* ctx, Call& c, const int64_t* crp, int32_t* ccol, void* cval_v) {
  using namespace cas;
  using AT = typename Acc<VIn>::T;
  AT* cval = static_cast<AT*>(cval_v);
  ctx->stats.split_rows = 0;
  int64_t off[kNumcBins + 1] = {0};
  for (int b = 0; b < kNumcBins; ++b) off[b + 1] = off[b] + c.numc_count[b];
  // bins in launch order, taken round-robin by the auxiliary streams.
  // bin_order 0 interleaves the bins of contended rows (dense and hash: many
  // products per output column, high cf) with the ESC bins (cf near 1), so
  // that each stream's neighbours run the other kind at the same time, the
  // GPU form of the reference's high- and low-contention thread groups
  // claiming morsels from the two ends of the cf-sorted queue
  // (src/ams/ams_utils.c:190-216, 697-736).  The default, bin_order 1,
  // launches the contended bins first and the ESC bins after them: never
  // slower on the R-MAT and Zipf inputs, 9% faster on G500 s17 ef8 when the
  // fused rows ended at 4800 products.
  const int interleaved[] = {kNB_Dense, kNB_E8K, kNB_H4K, kNB_E6K, kNB_E5K, kNB_E4K, kNB_E3K, kNB_H1K,
                             kNB_E2K, kNB_E1K, kNB_H256, kNB_Tiny};
  const int grouped[] = {kNB_Dense, kNB_H4K, kNB_H1K, kNB_H256, kNB_E8K, kNB_E6K, kNB_E5K, kNB_E4K,
                         kNB_E3K, kNB_E2K, kNB_E1K, kNB_Tiny};
  const int* order = ctx->bin_order == 1 ? grouped : interleaved;
  unsigned int* ovf_count = reinterpret_cast<unsigned int*>(ctx->d_counts + kSlotOvf);
  if (!c.ovf_preset) CAS_CUDA(ctx, cudaMemsetAsync(ovf_count, 0, sizeof(unsigned int), ctx->stream));
  CAS_TRY(fork(ctx));
  int64_t esc_rows = c.nf;  // fused rows may have handed rows to the radix-sort kernel too
  int si = 0;
  for (int oi = 0; oi < 12; ++oi) {
    const int b = order[oi];
    const int64_t n = c.numc_count[b];
    if (n == 0) continue;
    const int32_t* rows = c.rows + off[b];
    cudaStream_t s = ctx->profile ? ctx->stream : ctx->aux[si++ % kAux];  // profiling: one bin at a time
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_numc[0][b], s));
    const Csr& A = c.A.csr;
    const Csr& B = c.B.csr;
    switch (b) {
      case kNB_Tiny:
        k_numc_tiny<256, VIn><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(rows, n, A, B, crp, ccol, cval, ctx->d_status);
        break;
#define CAS_ESC_CASE(bin, CAP, NBB)                                                                      \
      case bin:                                                                                          \
        esc_rows += n;                                                                                   \
        launch_esc_bin<CAP, NBB, VIn>(ctx->esc_form, n, s, rows, A, B, c.b_sorted ? 1 : 0, crp, ccol, cval, \
                                      c.ovf, ovf_count, ctx->d_status);                                  \
        break;
      CAS_ESC_SHAPES(CAS_ESC_CASE)
#undef CAS_ESC_CASE
      case kNB_H256:
        k_numc_hash<256, 9, VIn><<<(unsigned)n, 256, smem_numc_hash<256, 9, VIn>(), s>>>(rows, A, B, crp, ccol, cval, ctx->d_status);
        break;
      case kNB_H1K:
        k_numc_hash<256, 11, VIn><<<(unsigned)n, 256, smem_numc_hash<256, 11, VIn>(), s>>>(rows, A, B, crp, ccol, cval, ctx->d_status);
        break;
      case kNB_H4K:
        k_numc_hash<512, 13, VIn><<<(unsigned)n, 512, smem_numc_hash<512, 13, VIn>(), s>>>(rows, A, B, crp, ccol, cval, ctx->d_status);
        break;
      case kNB_Dense: {
        if (!c.b_sorted && c.ncol > kRankCols)
          return set_err(ctx, CAS_ERR_BAD_INPUT, "heavy rows over more than %d columns need B rows sorted by column", kRankCols);
        // the rows of at least kSplitProducts products (log2 size classes kSplitLog2 and up) lead the
        // bin's heaviest-first order; they are split across blocks when their scratch fits
        int64_t n_split = 0;
        for (int k = 0; k <= kHeavyClasses - 1 - kSplitLog2; ++k) n_split += (int64_t)ctx->h_counts[kSlotHeavy + k];
        n_split = std::min(n_split, n);
        const int64_t max_slices = (c.ncol + kRankCols - 1) / kRankCols;
        n_split = std::min<int64_t>(n_split,
                                    (int64_t)((double)kSplitScratch * ctx->mem_share) / (max_slices * (kRankCols / 8)));
        if (!ctx->heavy_split) n_split = 0;
        ctx->stats.split_rows = n_split;
        if (n_split > 0) CAS_TRY(launch_heavy_split<VIn>(ctx, c, rows, n_split, crp, ccol, cval, s));
        if (n > n_split)
          k_numc_dense<512, VIn><<<(unsigned)(n - n_split), 512, smem_numc_dense<512, VIn>(), s>>>(
              rows + n_split, A, B, c.ncol, c.b_sorted ? 1 : 0, crp, ccol, cval, c.dbits, c.dslot, c.saved_slices,
              ctx->d_status);
        break;
      }
    }
    CAS_TRY(check_launch(ctx, "numeric bin"));
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_numc[1][b], s));
  }
  CAS_TRY(join(ctx));
  if (esc_rows > 0) {
    // rows whose columns bucket unevenly: radix-sort ESC, one persistent CTA per SM
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_ovf[0], ctx->stream));
    k_numc_esc_overflow<1024, 8192, VIn><<<(unsigned)std::min<int64_t>(esc_rows, ctx->sm_count), 1024,
                                          smem_numc_esc<1024, 8192, VIn>(), ctx->stream>>>(
        c.ovf, ovf_count, c.A.csr, c.B.csr, crp, ccol, cval, ctx->d_status);
    CAS_TRY(check_launch(ctx, "k_numc_esc_overflow"));
    if (ctx->profile) CAS_CUDA(ctx, cudaEventRecord(ctx->ev_ovf[1], ctx->stream));
    c.ovf_launched = true;
  }
  return CAS_OK;
}

int mode_of(cas_accum a) {
  return a == CAS_ACC_HASH ? cas::kAccHash : (a == CAS_ACC_HSERSC ? cas::kAccEsc : cas::kAccHybrid);
}

cas_status prepare(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, Call& c, double& h2d) {
  // launches are checked with cudaGetLastError, which also returns an error
  // another library in the process left behind; start from a clean slate
  cudaGetLastError();
  CAS_TRY(basic_checks(ctx, A, "A"));
  CAS_TRY(basic_checks(ctx, B, "B"));
  if (A->num_col != B->num_row)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "A is %lldx%lld but B has %lld rows", (long long)A->num_row,
                   (long long)A->num_col, (long long)B->num_row);
  if (A->val_type != B->val_type) return set_err(ctx, CAS_ERR_BAD_INPUT, "A and B have different value types");
  CAS_TRY(to_device(ctx, A, c.A, h2d));
  // B the same host matrix as A (C = A*A for a symmetric A, as for
  // C = A*A^T): one device copy serves both
  const bool alias = !A->on_device && !B->on_device && A->row_ptrs == B->row_ptrs && A->cols == B->cols &&
                     A->rats == B->rats && A->num_row == B->num_row && A->num_col == B->num_col &&
                     A->num_nnz == B->num_nnz && A->col_bytes == B->col_bytes;
  if (alias) {
    c.B.csr = c.A.csr;
    c.B.nnz = c.A.nnz;
    c.B.vt = c.A.vt;
  } else {
    CAS_TRY(to_device(ctx, B, c.B, h2d));
  }
  c.m = A->num_row;
  c.ncol = B->num_col;
  c.vt = A->val_type;
  return CAS_OK;
}

// C of one product in device memory (compute_dev).
struct DevC {
  int64_t* crp = nullptr;
  int32_t* ccol = nullptr;
  void* cval = nullptr;
  int64_t nnz = 0, nnz_known = 0;
};

void free_dev_c(DevC& o, cudaStream_t s) {
  if (o.crp) cudaFreeAsync(o.crp, s);
  if (o.ccol) cudaFreeAsync(o.ccol, s);
  if (o.cval) cudaFreeAsync(o.cval, s);
  o.crp = nullptr;
  o.ccol = nullptr;
  o.cval = nullptr;
}

// The four phases of one product whose A and B are on the device: C's row
// pointers, columns and values in device memory (o, nnz exact).  at_cap(cap)
// runs once C's bound is known and before NUMC is launched (a host output
// takes its blocks there, while the GPU works).  The phase boundaries are
// recorded on ev_phase[0..4].
template <typename F>
cas_status compute_dev(cas_ctx* ctx, cas_accum accum, Call& c, bool validate, DevC& o, F&& at_cap) {
  using namespace cas;
  const size_t vbytes = 8;  // fp64 or int64 output
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_phase[0], ctx->stream));
  // INIT
  CAS_TRY(phase_init(ctx, c, validate));
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_phase[1], ctx->stream));
  // SYMB
  CAS_TRY(dev_alloc(ctx, (void**)&o.crp, sizeof(int64_t) * (c.m + 1)));
  CAS_TRY(launch_symb_bins(ctx, c, c.row_nz));
  CAS_TRY(launch_scan(ctx, o.crp, c.row_nz, c.m + 1, c.partial,
                      reinterpret_cast<int64_t*>(ctx->d_counts + kSlotNnz)));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotNnz, ctx->d_counts + kSlotNnz, 1, ctx->stream));
  CAS_TRY(check_status(ctx));
  // counts of the rows that had a symbolic pass; the fused rows add theirs
  // in NUMC, within the bound min(products, columns) each
  o.nnz_known = (int64_t)ctx->h_counts[kSlotNnz];
  o.nnz = o.nnz_known;
  const int64_t cap = o.nnz_known + (c.nf > 0 ? c.f_bound : 0);
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_phase[2], ctx->stream));
  // MGMT
  CAS_TRY(dev_alloc(ctx, (void**)&o.ccol, sizeof(int32_t) * cap));
  CAS_TRY(dev_alloc(ctx, &o.cval, vbytes * cap));
  CAS_TRY(at_cap(cap));
  CAS_TRY(numc_bins(ctx, c, o.crp, mode_of(accum)));
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_phase[3], ctx->stream));
  // NUMC: the fused rows first (they place themselves after the known
  // counts), then the scan of all counts, which the other kernels write by
  if (c.nf > 0) {
    if (c.vt == CAS_VAL_F64) CAS_TRY(launch_fused<double>(ctx, c, o.crp, o.ccol, o.cval, cap));
    else CAS_TRY(launch_fused<int32_t>(ctx, c, o.crp, o.ccol, o.cval, cap));
    CAS_TRY(launch_scan(ctx, o.crp, c.row_nz, c.m + 1, c.partial,
                        reinterpret_cast<int64_t*>(ctx->d_counts + kSlotNnz)));
  }
  if (c.vt == CAS_VAL_F64) CAS_TRY(launch_numc_bins<double>(ctx, c, o.crp, o.ccol, o.cval));
  else CAS_TRY(launch_numc_bins<int32_t>(ctx, c, o.crp, o.ccol, o.cval));
  CAS_TRY(scratch_free(ctx, c));
  CAS_CUDA(ctx, cudaEventRecord(ctx->ev_phase[4], ctx->stream));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotOvf, ctx->d_counts + kSlotOvf, 1, ctx->stream));
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotNnz, ctx->d_counts + kSlotNnz, 1, ctx->stream));
  CAS_TRY(check_status(ctx));
  o.nnz = (int64_t)ctx->h_counts[kSlotNnz];
  return CAS_OK;
}

// The counters of one product just computed (its phases' events and counts
// are still in the context); kernel launches and copied bytes are the
// caller's.
cas_stats product_stats(cas_ctx* ctx, const Call& c, const DevC& o) {
  using namespace cas;
  cas_stats s{};
  s.flop = c.flop;
  s.max_row_flp = c.max_flp;
  s.nnz_c = o.nnz;
  for (int b = 0; b < kSymbBins; ++b) s.symb_bin_rows[b] = c.symb_count[b];
  for (int b = 0; b < kNumcBins; ++b) s.numc_bin_rows[b] = c.numc_count[b];
  const double vin = c.vt == CAS_VAL_F64 ? 8.0 : 4.0;
  for (int b = 0; b < kNumcBins; ++b) {
    const double flp = (double)ctx->h_counts[kSlotBinSums + b];
    const double nzc = (double)ctx->h_counts[kSlotBinSums + kNumcBins + b];
    const double nza = (double)ctx->h_counts[kSlotBinSums + 2 * kNumcBins + b];
    s.numc_bin_flop[b] = (int64_t)ctx->h_counts[kSlotBinSums + b];
    s.numc_bin_nnz[b] = (int64_t)nzc;
    s.numc_bin_bytes[b] = (4 + vin) * (nza + flp) + 12.0 * nzc + 16.0 * (double)c.numc_count[b];
    float ms = 0;
    if (ctx->profile && b != kNB_Zero && c.numc_count[b] > 0 &&
        cudaEventElapsedTime(&ms, ctx->ev_numc[0][b], ctx->ev_numc[1][b]) == cudaSuccess)
      s.numc_bin_ms[b] = ms;
  }
  s.fused_rows = c.nf;
  s.fused_flop = c.f_flop;
  if (c.nf > 0) {
    // nnz(C) of the fused rows: all entries less those of the rows with a symbolic pass
    s.fused_bytes = (4 + vin) * ((double)c.f_nnza + (double)c.f_flop) + 12.0 * (double)(o.nnz - o.nnz_known) +
                    16.0 * (double)c.nf;
    float ms = 0;
    if (ctx->profile && cudaEventElapsedTime(&ms, ctx->ev_fused[0], ctx->ev_fused[1]) == cudaSuccess) s.fused_ms = ms;
  }
  s.esc_overflow_rows = (int64_t)(ctx->h_counts[kSlotOvf] & 0xFFFFFFFFull);
  {
    float ms = 0;
    if (ctx->profile && c.ovf_launched && cudaEventElapsedTime(&ms, ctx->ev_ovf[0], ctx->ev_ovf[1]) == cudaSuccess)
      s.esc_overflow_ms = ms;
  }
  for (int b = 0; b < kSymbBins; ++b) {
    float ms = 0;
    if (ctx->profile && b != kSB_Zero && c.symb_count[b] > 0 &&
        cudaEventElapsedTime(&ms, ctx->ev_symb[0][b], ctx->ev_symb[1][b]) == cudaSuccess)
      s.symb_bin_ms[b] = ms;
  }
  s.split_rows = ctx->stats.split_rows;  // set by this product's launch_numc_bins
  s.out_blocks = 1;
  cudaGetLastError();  // leave no error pending from the timing queries
  return s;
}

// a += b for the counters of two row blocks of one product
void add_stats(cas_stats& a, const cas_stats& b) {
  a.flop += b.flop;
  a.max_row_flp = std::max(a.max_row_flp, b.max_row_flp);
  a.nnz_c += b.nnz_c;
  for (int i = 0; i < CAS_SYMB_BINS; ++i) {
    a.symb_bin_rows[i] += b.symb_bin_rows[i];
    a.symb_bin_ms[i] += b.symb_bin_ms[i];
  }
  for (int i = 0; i < CAS_NUMC_BINS; ++i) {
    a.numc_bin_rows[i] += b.numc_bin_rows[i];
    a.numc_bin_ms[i] += b.numc_bin_ms[i];
    a.numc_bin_bytes[i] += b.numc_bin_bytes[i];
    a.numc_bin_flop[i] += b.numc_bin_flop[i];
    a.numc_bin_nnz[i] += b.numc_bin_nnz[i];
  }
  a.esc_overflow_rows += b.esc_overflow_rows;
  a.esc_overflow_ms += b.esc_overflow_ms;
  a.fused_rows += b.fused_rows;
  a.fused_flop += b.fused_flop;
  a.fused_bytes += b.fused_bytes;
  a.fused_ms += b.fused_ms;
  a.split_rows += b.split_rows;
  a.out_blocks += b.out_blocks;
}

void phase_times(cas_ctx* ctx, double t[4]) {
  for (int i = 0; i < 4; ++i) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ctx->ev_phase[i], ctx->ev_phase[i + 1]) == cudaSuccess) t[i] += ms * 1e-3;
  }
  cudaGetLastError();
}

// The sum over A's rows of min(products, columns), an upper bound on nnz(C).
cas_status nnz_bound(cas_ctx* ctx, const Call& c, int64_t& bound) {
  using namespace cas;
  unsigned long long* d = ctx->d_counts + kSlotNnz;
  CAS_CUDA(ctx, cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream));
  if (c.m > 0) {
    k_nnz_bound<256><<<grid_for(c.m * 32, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(c.A.csr, c.B.csr, c.ncol, d);
    CAS_TRY(check_launch(ctx, "k_nnz_bound"));
  }
  CAS_TRY(fetch_words(ctx, ctx->h_counts_dev + kSlotNnz, d, 1, ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  bound = (int64_t)ctx->h_counts[kSlotNnz];
  return CAS_OK;
}

// C in host memory by row blocks of about equal A entries.  Each block runs
// the four phases as a product of its own (with its own fused-row tickets)
// into device memory; its row pointers are moved to its place in C, and the
// block is copied out on the copy stream, straight into C's host arrays where
// the context has registered them, while the next block is computed.  The
// host arrays are sized by `bound` (the sum over rows of min(products,
// columns)); num_nnz is exact.
cas_status run_blocked(cas_ctx* ctx, cas_accum accum, const cas_csr* A, Call& full, int nblk, int64_t bound,
                       cas_csr* C, cas_runtime* rt, double& d2h) {
  using namespace cas;
  const size_t vbytes = 8;
  const int64_t m = full.m;
  std::vector<int64_t> rb((size_t)nblk + 1);
  for (int k = 0; k <= nblk; ++k) {
    if (!A->on_device) {
      const int64_t target = (int64_t)((double)A->num_nnz * k / nblk);
      rb[(size_t)k] = std::lower_bound(A->row_ptrs, A->row_ptrs + m + 1, target) - A->row_ptrs;
    } else {
      rb[(size_t)k] = m * k / nblk;
    }
  }
  rb[0] = 0;
  rb[(size_t)nblk] = m;
  int64_t* h_rp = static_cast<int64_t*>(host_take(ctx, sizeof(int64_t) * (m + 1)));
  void* h_col = host_take(ctx, sizeof(int32_t) * (size_t)(bound > 0 ? bound : 1));
  void* h_val = host_take(ctx, vbytes * (size_t)(bound > 0 ? bound : 1));
  auto free_host = [&] {
    host_give(ctx, h_rp);
    host_give(ctx, h_col);
    host_give(ctx, h_val);
  };
  if (!h_rp || !h_col || !h_val) {
    free_host();
    return set_err(ctx, CAS_ERR_OOM, "host allocation of C failed");
  }
  const bool pin_col = host_is_pinned(ctx, h_col), pin_val = host_is_pinned(ctx, h_val);
  // C's row pointers gather on the device, each block's moved to its place,
  // and go out in one copy at the end
  int64_t* d_rp = nullptr;
  {
    const cas_status a = dev_alloc(ctx, (void**)&d_rp, sizeof(int64_t) * (size_t)(m + 1));
    if (a != CAS_OK) {
      free_host();
      return a;
    }
  }
  cudaEvent_t ev_done = nullptr;
  CAS_CUDA(ctx, cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
  // A block's device buffers are freed (on the main stream) only once its
  // copies are seen to be complete: freed in the copy stream's order, the
  // pool could hand their memory to a later block and make the main stream
  // wait for the copy, which would serialise computing and copying.
  struct InFlight {
    DevC o;
    cudaEvent_t copied;
  };
  std::deque<InFlight> inflight;
  auto reap = [&](bool wait) {
    while (!inflight.empty()) {
      InFlight& f = inflight.front();
      if (wait) cudaEventSynchronize(f.copied);
      else if (cudaEventQuery(f.copied) != cudaSuccess) break;
      free_dev_c(f.o, ctx->stream);
      cudaEventDestroy(f.copied);
      inflight.pop_front();
    }
    cudaGetLastError();  // a not-ready query leaves no error behind
  };
  cas_stats acc{};
  double t[4] = {0, 0, 0, 0};
  int64_t base = 0;
  int nrun = 0;
  cas_status st = CAS_OK;
  for (int k = 0; k < nblk && st == CAS_OK; ++k) {
    const int64_t r0 = rb[(size_t)k], r1 = rb[(size_t)k + 1];
    if (r1 <= r0) continue;
    Call ck;
    ck.A.csr = full.A.csr;
    ck.A.csr.rp = full.A.csr.rp + r0;
    ck.A.csr.nrow = r1 - r0;
    ck.A.nnz = full.A.nnz;
    ck.A.vt = full.A.vt;
    ck.B.csr = full.B.csr;
    ck.B.nnz = full.B.nnz;
    ck.B.vt = full.B.vt;
    ck.m = r1 - r0;
    ck.ncol = full.ncol;
    ck.vt = full.vt;
    ck.fuse = full.fuse;
    ck.b_sorted = full.b_sorted;
    DevC o;
    st = compute_dev(ctx, accum, ck, false, o, [](int64_t) { return CAS_OK; });
    if (st == CAS_OK && o.nnz > bound - base)
      st = set_err(ctx, CAS_ERR_DEVICE, "row block %d: %lld entries past the output bound", k,
                   (long long)(base + o.nnz - bound));
    if (st == CAS_OK) {
      k_rebase_to<<<grid_for(ck.m + 1, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(d_rp + r0, o.crp, ck.m + 1,
                                                                                        base);
      st = check_launch(ctx, "k_rebase_to");
    }
    if (st != CAS_OK) {
      scratch_free(ctx, ck);
      free_dev_c(o, ctx->stream);
      break;
    }
    phase_times(ctx, t);
    const cas_stats bs = product_stats(ctx, ck, o);
    if (nrun == 0) acc = bs;
    else add_stats(acc, bs);
    ++nrun;
    // the block's columns and values: arrays the context has not registered
    // through the staging buffers now, the others by DMA on the copy stream
    char* col_dst = static_cast<char*>(h_col) + sizeof(int32_t) * (size_t)base;
    char* val_dst = static_cast<char*>(h_val) + vbytes * (size_t)base;
    const size_t col_b = sizeof(int32_t) * (size_t)o.nnz, val_b = vbytes * (size_t)o.nnz;
    if (!pin_col && st == CAS_OK) st = d2h_staged(ctx, col_dst, o.ccol, col_b);
    if (!pin_val && st == CAS_OK) st = d2h_staged(ctx, val_dst, o.cval, val_b);
    bool queued = false;  // the copy stream waits for the block and reads its buffers
    if (st == CAS_OK) {
      cudaError_t e = cudaEventRecord(ev_done, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, ev_done, 0);
      queued = e == cudaSuccess;
      if (e == cudaSuccess && pin_col && col_b)
        e = cudaMemcpyAsync(col_dst, o.ccol, col_b, cudaMemcpyDeviceToHost, ctx->copy_stream);
      if (e == cudaSuccess && pin_val && val_b)
        e = cudaMemcpyAsync(val_dst, o.cval, val_b, cudaMemcpyDeviceToHost, ctx->copy_stream);
      if (e != cudaSuccess) st = set_err(ctx, CAS_ERR_CUDA, "copy of row block %d: %s", k, cudaGetErrorString(e));
      ctx->d2h_direct += (pin_col ? (double)col_b : 0.0) + (pin_val ? (double)val_b : 0.0);
    }
    cudaEvent_t copied = nullptr;
    if (queued && cudaEventCreateWithFlags(&copied, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventRecord(copied, ctx->copy_stream) == cudaSuccess) {
      inflight.push_back({o, copied});
    } else {
      if (copied) cudaEventDestroy(copied);
      if (queued) cudaStreamSynchronize(ctx->copy_stream);
      free_dev_c(o, ctx->stream);
    }
    reap(false);
    d2h += (double)(col_b + val_b);
    base += o.nnz;
  }
  const cudaError_t ce = cudaStreamSynchronize(ctx->copy_stream);
  reap(true);
  cudaEventDestroy(ev_done);
  if (st == CAS_OK && ce != cudaSuccess)
    st = set_err(ctx, CAS_ERR_CUDA, "copy of C's row blocks: %s", cudaGetErrorString(ce));
  if (st == CAS_OK) {
    st = d2h_out(ctx, h_rp, d_rp, sizeof(int64_t) * (size_t)(m + 1));
    d2h += sizeof(int64_t) * (double)(m + 1);
  }
  cudaFreeAsync(d_rp, ctx->stream);
  if (st == CAS_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    st = set_err(ctx, CAS_ERR_CUDA, "row blocks: %s", cudaGetErrorString(cudaGetLastError()));
  if (st != CAS_OK) {
    free_host();
    return st;
  }
  C->num_row = m;
  C->num_col = full.ncol;
  C->num_nnz = base;
  C->val_type = full.vt;
  C->owned = 2;
  C->on_device = 0;
  C->col_bytes = 4;
  C->row_ptrs = h_rp;
  C->cols = h_col;
  C->rats = h_val;
  if (rt) {
    rt->init_time = t[0];
    rt->symb_time = t[1];
    rt->mgmt_time = t[2];
    rt->numc_time = t[3];
    rt->total_time = t[0] + t[1] + t[2] + t[3];
  }
  ctx->stats = acc;
  return CAS_OK;
}

cas_status run_spgemm(cas_ctx* ctx, cas_accum accum, const cas_csr* A, const cas_csr* B, cas_csr* C,
                      cas_runtime* rt) {
  using namespace cas;
  Call c;
  double h2d = 0, d2h = 0;
  ctx->d2h_direct = 0;
  const bool c_on_device = C->on_device != 0;
  const int c_col_bytes = c_on_device ? 4 : (C->col_bytes == 8 ? 8 : 4);
  CAS_TRY(prepare(ctx, A, B, c, h2d));
  memset(C, 0, sizeof(*C));
  c.fuse = ctx->fuse && accum != CAS_ACC_HASH ? ctx->fused_lo : 0;
  const size_t vbytes = 8;  // fp64 or int64 output
  auto finish = [&](cas_status st) -> cas_status {
    cas_status f1 = free_owned(ctx, c.A), f2 = free_owned(ctx, c.B);
    if (st == CAS_OK) st = f1 != CAS_OK ? f1 : f2;
    if (st == CAS_OK) {
      cas_stats& s = ctx->stats;
      s.kernel_launches = ctx->launches;
      s.h2d_bytes = h2d;
      s.d2h_bytes = d2h;
      s.d2h_direct_bytes = ctx->d2h_direct;
    }
    return st;
  };
  // a large C in host memory with int32 columns goes by row blocks, each
  // copied out while the next is computed (cas_tuning.out_blocks)
  bool checked = false;
  if (!c_on_device && c_col_bytes == 4 && ctx->out_blocks != 1 && c.m > 1) {
    cas_status st = check_inputs(ctx, c);
    int64_t bound = 0;
    if (st == CAS_OK) st = nnz_bound(ctx, c, bound);
    if (st != CAS_OK) return finish(st);
    checked = true;
    int64_t nblk = ctx->out_blocks;
    if (nblk == 0) {
      const double bytes = (4.0 + (double)vbytes) * (double)bound;
      nblk = bytes < kOutBlockMin ? 1
                                  : (int64_t)std::min(std::max(2.0, std::ceil(bytes / kOutBlockBytes)), (double)kMaxOutBlocks);
    }
    nblk = std::min(nblk, c.m);
    if (nblk > 1) return finish(run_blocked(ctx, accum, A, c, (int)nblk, bound, C, rt, d2h));
  }
  DevC o;
  int64_t* h_rp = nullptr;
  void *h_col = nullptr, *h_val = nullptr;
  auto free_host = [&] {
    host_give(ctx, h_rp);
    host_give(ctx, h_col);
    host_give(ctx, h_val);
  };
  cas_status st = compute_dev(ctx, accum, c, !checked, o, [&](int64_t cap) -> cas_status {
    if (c_on_device) return CAS_OK;
    h_rp = static_cast<int64_t*>(host_take(ctx, sizeof(int64_t) * (c.m + 1)));
    h_col = host_take(ctx, (size_t)c_col_bytes * (size_t)(cap > 0 ? cap : 1));
    h_val = host_take(ctx, vbytes * (size_t)(cap > 0 ? cap : 1));
    if (!h_rp || !h_col || !h_val) return set_err(ctx, CAS_ERR_OOM, "host allocation of C failed");
    return CAS_OK;
  });
  if (st != CAS_OK) {
    free_host();
    scratch_free(ctx, c);
    free_dev_c(o, ctx->stream);
    return finish(st);
  }
  const int64_t nnz = o.nnz;
  C->num_row = c.m;
  C->num_col = c.ncol;
  C->num_nnz = nnz;
  C->val_type = c.vt;
  C->owned = 1;
  if (c_on_device) {
    C->on_device = 1;
    C->col_bytes = 4;
    C->row_ptrs = o.crp;
    C->cols = o.ccol;
    C->rats = o.cval;
  } else {
    C->owned = 2;
    C->on_device = 0;
    C->col_bytes = c_col_bytes;
    C->row_ptrs = h_rp;
    C->cols = h_col;
    C->rats = h_val;
    cas_status cs = d2h_out(ctx, C->row_ptrs, o.crp, sizeof(int64_t) * (c.m + 1));
    if (cs == CAS_OK) cs = d2h_out(ctx, C->rats, o.cval, vbytes * nnz);
    if (cs == CAS_OK) cs = d2h_out(ctx, C->cols, o.ccol, sizeof(int32_t) * nnz, c_col_bytes == 8);
    d2h += sizeof(int64_t) * (double)(c.m + 1) + (vbytes + c_col_bytes) * (double)nnz;
    free_dev_c(o, ctx->stream);
    if (cs == CAS_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      cs = set_err(ctx, CAS_ERR_CUDA, "copy of C: %s", cudaGetErrorString(cudaGetLastError()));
    if (cs != CAS_OK) {
      free_host();
      memset(C, 0, sizeof(*C));
      return finish(cs);
    }
  }
  if (rt) {
    double t[4] = {0, 0, 0, 0};
    phase_times(ctx, t);
    rt->init_time = t[0];
    rt->symb_time = t[1];
    rt->mgmt_time = t[2];
    rt->numc_time = t[3];
    rt->total_time = t[0] + t[1] + t[2] + t[3];
  }
  ctx->stats = product_stats(ctx, c, o);
  return finish(CAS_OK);
}

}  // namespace

// ================================================================= C ABI
extern "C" {

cas_status cas_create(int device, cas_ctx** out) {
  if (!out) return CAS_ERR_BAD_INPUT;
  *out = nullptr;
  cas_ctx* ctx = new (std::nothrow) cas_ctx();
  if (!ctx) return CAS_ERR_OOM;
  ctx->device = device;
  cas_status st = [&]() -> cas_status {
    CAS_CUDA(ctx, cudaSetDevice(device));
    CAS_CUDA(ctx, cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
    CAS_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
    ctx->stream = ctx->own_stream;
    for (int i = 0; i < kAux; ++i) {
      CAS_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->aux[i], cudaStreamNonBlocking));
      CAS_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming));
    }
    CAS_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CAS_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 5; ++i) CAS_CUDA(ctx, cudaEventCreate(&ctx->ev_phase[i]));
    for (int i = 0; i < 2; ++i) CAS_CUDA(ctx, cudaEventCreate(&ctx->ev_fused[i]));
    for (int i = 0; i < 2; ++i) {
      CAS_CUDA(ctx, cudaEventCreate(&ctx->ev_ovf[i]));
      for (int b = 0; b < cas::kSymbBins; ++b) CAS_CUDA(ctx, cudaEventCreate(&ctx->ev_symb[i][b]));
      for (int b = 0; b < cas::kNumcBins; ++b) CAS_CUDA(ctx, cudaEventCreate(&ctx->ev_numc[i][b]));
    }
    CAS_CUDA(ctx, cudaMalloc(&ctx->d_status, sizeof(cas::DevStatus)));
    CAS_CUDA(ctx, cudaMalloc(&ctx->d_counts, sizeof(unsigned long long) * kCountSlots));
    CAS_CUDA(ctx, cudaMallocHost(&ctx->h_counts, sizeof(unsigned long long) * kCountSlots));
    CAS_CUDA(ctx, cudaMallocHost(&ctx->h_status, sizeof(cas::DevStatus)));
    CAS_CUDA(ctx, cudaMallocHost(&ctx->h_misc, sizeof(unsigned long long) * kMiscWords));
    CAS_CUDA(ctx, cudaHostGetDevicePointer((void**)&ctx->h_counts_dev, ctx->h_counts, 0));
    CAS_CUDA(ctx, cudaHostGetDevicePointer((void**)&ctx->h_status_dev, ctx->h_status, 0));
    CAS_CUDA(ctx, cudaHostGetDevicePointer((void**)&ctx->h_misc_dev, ctx->h_misc, 0));
    // keep freed device memory in the stream-ordered pool between calls
    cudaMemPool_t pool;
    CAS_CUDA(ctx, cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thresh = UINT64_MAX;
    CAS_CUDA(ctx, cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
    CAS_TRY(setup_kernels(ctx));
    return CAS_OK;
  }();
  if (st != CAS_OK) {
    fprintf(stderr, "cas_create: %s\n", ctx->err.c_str());
    cas_destroy(ctx);
    return st;
  }
  *out = ctx;
  return CAS_OK;
}

void cas_destroy(cas_ctx* ctx) {
  if (!ctx) return;
  for (cas_ctx* w : ctx->batch_workers) cas_destroy(w);
  ctx->batch_workers.clear();
  cudaSetDevice(ctx->device);
  if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  for (int i = 0; i < kAux; ++i) {
    if (ctx->aux[i]) cudaStreamDestroy(ctx->aux[i]);
    if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  for (int i = 0; i < 5; ++i)
    if (ctx->ev_phase[i]) cudaEventDestroy(ctx->ev_phase[i]);
  for (int i = 0; i < 2; ++i)
    if (ctx->ev_fused[i]) cudaEventDestroy(ctx->ev_fused[i]);
  for (int i = 0; i < 2; ++i) {
    if (ctx->ev_ovf[i]) cudaEventDestroy(ctx->ev_ovf[i]);
    for (int b = 0; b < cas::kSymbBins; ++b)
      if (ctx->ev_symb[i][b]) cudaEventDestroy(ctx->ev_symb[i][b]);
    for (int b = 0; b < cas::kNumcBins; ++b)
      if (ctx->ev_numc[i][b]) cudaEventDestroy(ctx->ev_numc[i][b]);
  }
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->d_counts) cudaFree(ctx->d_counts);
  if (ctx->h_counts) cudaFreeHost(ctx->h_counts);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->h_misc) cudaFreeHost(ctx->h_misc);
  for (int i = 0; i < kStageBufs; ++i) {
    if (ctx->h_stage[i]) cudaFreeHost(ctx->h_stage[i]);
    if (ctx->ev_stage[i]) cudaEventDestroy(ctx->ev_stage[i]);
  }
  {
    // blocks still held by callers stay valid host memory, no longer
    // registered and no longer recorded: cas_csr_free then just frees them
    std::lock_guard<std::mutex> lock(g_host_mu);
    for (void* p : ctx->host_pinned) {
      cudaHostUnregister(p);
      g_pinned_bytes.fetch_sub(pin_length(ctx->host_blocks[p]));
    }
    for (auto& b : ctx->host_blocks) g_host_owner.erase(b.first);
    for (auto& b : ctx->host_free) free(b.first);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

cas_status cas_set_stream(cas_ctx* ctx, void* stream) {
  if (!ctx) return CAS_ERR_BAD_INPUT;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return CAS_OK;
}

cas_status cas_set_acc_thres(cas_ctx* ctx, double thres) {
  if (!ctx || !(thres >= 0.0)) return CAS_ERR_BAD_INPUT;
  ctx->acc_thres = thres;
  return CAS_OK;
}

const char* cas_last_error(const cas_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

cas_status cas_set_tuning(cas_ctx* ctx, const cas_tuning* t) {
  if (!ctx || !t) return CAS_ERR_BAD_INPUT;
  if (!(t->acc_thres >= 0.0) || t->fused_min_products < 32 || t->fused_min_products >= (int)cas::kFusedHi ||
      t->esc_max_products < 32 || t->esc_max_products > 8192 || t->hash_max_nnz < 0 || t->hash_max_nnz > 4096 ||
      t->esc_form < 0 || t->esc_form > 2 || (t->heavy_split != 0 && t->heavy_split != 1) ||
      (t->bin_order != 0 && t->bin_order != 1) || t->out_blocks < 0 || t->out_blocks > kMaxOutBlocks)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "tuning out of range");
  ctx->acc_thres = t->acc_thres;
  ctx->fuse = t->fusion != 0;
  ctx->fused_lo = t->fused_min_products;
  ctx->esc_max = t->esc_max_products;
  ctx->hash_max = t->hash_max_nnz;
  ctx->esc_form = t->esc_form;
  ctx->heavy_split = t->heavy_split != 0;
  ctx->bin_order = t->bin_order;
  ctx->out_blocks = t->out_blocks;
  return CAS_OK;
}

cas_status cas_get_tuning(const cas_ctx* ctx, cas_tuning* t) {
  if (!ctx || !t) return CAS_ERR_BAD_INPUT;
  t->acc_thres = ctx->acc_thres;
  t->fusion = ctx->fuse ? 1 : 0;
  t->fused_min_products = ctx->fused_lo;
  t->esc_max_products = ctx->esc_max;
  t->hash_max_nnz = ctx->hash_max;
  t->esc_form = ctx->esc_form;
  t->heavy_split = ctx->heavy_split ? 1 : 0;
  t->bin_order = ctx->bin_order;
  t->out_blocks = ctx->out_blocks;
  return CAS_OK;
}

cas_status cas_set_fusion(cas_ctx* ctx, int on) {
  if (!ctx) return CAS_ERR_BAD_INPUT;
  ctx->fuse = on != 0;
  return CAS_OK;
}

cas_status cas_set_profiling(cas_ctx* ctx, int on) {
  if (!ctx) return CAS_ERR_BAD_INPUT;
  ctx->profile = on != 0;
  return CAS_OK;
}

cas_status cas_get_stats(const cas_ctx* ctx, cas_stats* out) {
  if (!ctx || !out) return CAS_ERR_BAD_INPUT;
  *out = ctx->stats;
  out->kernel_launches = ctx->launches;
  return CAS_OK;
}

cas_status cas_spgemm(cas_ctx* ctx, cas_accum accum, const cas_csr* A, const cas_csr* B, cas_csr* C,
                      cas_runtime* rt) {
  if (!ctx || !C) return CAS_ERR_BAD_INPUT;
  if (accum != CAS_ACC_HASH && accum != CAS_ACC_HSERSC && accum != CAS_ACC_HYBACC)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "unknown accumulator %d", (int)accum);
  CAS_CUDA(ctx, cudaSetDevice(ctx->device));
  return run_spgemm(ctx, accum, A, B, C, rt);
}

cas_status cas_csr_free(cas_ctx* ctx, cas_csr* C) {
  if (!C) return CAS_ERR_BAD_INPUT;
  if (C->owned) {
    if (C->on_device) {
      if (ctx) {
        cudaStream_t s = ctx->stream;
        cudaFreeAsync(C->row_ptrs, s);
        cudaFreeAsync(C->cols, s);
        cudaFreeAsync(C->rats, s);
        cudaStreamSynchronize(s);
      } else {
        cudaFree(C->row_ptrs);
        cudaFree(C->cols);
        cudaFree(C->rats);
      }
    } else {
      // owned 2: blocks of a context's host cache; host_give finds their owner
      host_give(ctx, C->row_ptrs);
      host_give(ctx, C->cols);
      host_give(ctx, C->rats);
    }
  }
  memset(C, 0, sizeof(*C));
  return CAS_OK;
}

// ---- phase functions ---------------------------------------------------

cas_status cas_flp_populate(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, int64_t* d_row_flp) {
  if (!ctx || !d_row_flp) return CAS_ERR_BAD_INPUT;
  if (!A || !B || !A->on_device || !B->on_device)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "phase functions take device matrices");
  Call c;
  double h2d = 0;
  CAS_TRY(prepare(ctx, A, B, c, h2d));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_counts, 0, sizeof(unsigned long long) * kCountSlots, ctx->stream));
  CAS_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(cas::DevStatus), ctx->stream));
  if (c.m > 0) {
    cas::k_flp<256><<<grid_for(c.m * 32, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        c.A.csr, c.B.csr, c.ncol, d_row_flp, ctx->d_counts + kSlotTotals, ctx->d_counts + kSlotSymb, ctx->d_status,
        0, ctx->d_counts + kSlotFused);
    CAS_TRY(check_launch(ctx, "k_flp"));
  }
  return check_status(ctx);
}

cas_status cas_scan(cas_ctx* ctx, int64_t* d_out, const int64_t* d_in, int64_t n) {
  if (!ctx || !d_out || (n > 1 && !d_in) || n < 0) return CAS_ERR_BAD_INPUT;
  if (n == 0) return CAS_OK;
  const int64_t nparts = (n + cas::kScanTile - 1) / cas::kScanTile;
  int64_t* partial = nullptr;
  CAS_TRY(dev_alloc(ctx, (void**)&partial, sizeof(int64_t) * (nparts + 1)));
  cas_status st = launch_scan(ctx, d_out, d_in, n, partial, nullptr);
  CAS_CUDA(ctx, cudaFreeAsync(partial, ctx->stream));
  CAS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

cas_status cas_hash_symb(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, const int64_t* d_row_flp,
                         int64_t* d_row_nz) {
  if (!ctx || !d_row_nz) return CAS_ERR_BAD_INPUT;
  if (!A || !B || !A->on_device || !B->on_device)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "phase functions take device matrices");
  (void)d_row_flp;  // recomputed together with the bins
  Call c;
  double h2d = 0;
  CAS_TRY(prepare(ctx, A, B, c, h2d));
  CAS_TRY(phase_init(ctx, c, true));
  CAS_TRY(launch_symb_bins(ctx, c, d_row_nz));
  CAS_TRY(scratch_free(ctx, c));
  return check_status(ctx);
}

static cas_status numc_entry(cas_ctx* ctx, cas_accum accum, const cas_csr* A, const cas_csr* B, cas_csr* C) {
  if (!ctx || !C) return CAS_ERR_BAD_INPUT;
  if (!A || !B || !A->on_device || !B->on_device || !C->on_device)
    return set_err(ctx, CAS_ERR_BAD_INPUT, "phase functions take device matrices");
  Call c;
  double h2d = 0;
  CAS_TRY(prepare(ctx, A, B, c, h2d));
  CAS_TRY(phase_init(ctx, c, true));
  CAS_TRY(numc_bins(ctx, c, C->row_ptrs, mode_of(accum)));
  if (c.vt == CAS_VAL_F64)
    CAS_TRY(launch_numc_bins<double>(ctx, c, C->row_ptrs, static_cast<int32_t*>(C->cols), C->rats));
  else
    CAS_TRY(launch_numc_bins<int32_t>(ctx, c, C->row_ptrs, static_cast<int32_t*>(C->cols), C->rats));
  CAS_TRY(scratch_free(ctx, c));
  return check_status(ctx);
}

cas_status cas_hash_numc(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, const int64_t* d_row_flp, cas_csr* C) {
  (void)d_row_flp;
  return numc_entry(ctx, CAS_ACC_HASH, A, B, C);
}
cas_status cas_hsersc_numc(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, const int64_t* d_row_flp, cas_csr* C) {
  (void)d_row_flp;
  return numc_entry(ctx, CAS_ACC_HSERSC, A, B, C);
}
cas_status cas_hybacc_numc(cas_ctx* ctx, const cas_csr* A, const cas_csr* B, const int64_t* d_row_flp, cas_csr* C) {
  (void)d_row_flp;
  return numc_entry(ctx, CAS_ACC_HYBACC, A, B, C);
}

}  // extern "C"

// ============================================= digests and batches of products
#include "cas_batch.cu"
#include "cas_serve.cu"
#include "cas_transpose.cu"

// ===================================================== scan without allocation
// cas_scan_noalloc: the same exclusive scan as cas_scan, for callers that must
// not allocate device memory — for example a process whose device memory is
// handed out by another framework's pool and budget, where a cudaMalloc behind
// its back breaks the accounting, or a latency-sensitive loop that cannot take
// the device-wide synchronisation a cudaMalloc or cudaFree may imply.  The
// per-tile partial sums live in a fixed array in device memory, created when
// the library is loaded and kept by every device that loads it until the
// process exits (kNoAllocParts partials, 128 KiB).  Every call overwrites the
// partials it reads before reading them, so nothing needs clearing, and calls
// that overlap on the GPU (on different streams, or from several host threads)
// share the array and race: serialise them.  The array's device address is
// looked up once per device and kept; after cudaDeviceReset (or any teardown
// of the device's primary context) it is stale, so the function must not be
// used again in that process.
namespace {

constexpr int64_t kNoAllocParts = 16384;  // scans of up to kNoAllocParts * kScanTile elements
constexpr int kNoAllocMaxDevices = 256;

static __device__ __align__(256) int64_t g_noalloc_partials[kNoAllocParts];

std::mutex g_noalloc_mu;
int64_t* g_noalloc_addr[kNoAllocMaxDevices] = {};

}  // namespace

extern "C" cas_status cas_scan_noalloc(int64_t* d_out, const int64_t* d_in, int64_t n, void* stream) {
  if (!d_out || n < 0 || (n > 1 && !d_in)) return CAS_ERR_BAD_INPUT;
  if (n == 0) return CAS_OK;
  const int64_t nparts = (n + cas::kScanTile - 1) / cas::kScanTile;
  if (nparts > kNoAllocParts) return CAS_ERR_REJECTED;  // n > kNoAllocParts * kScanTile
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return CAS_ERR_CUDA;
  int64_t* partial = nullptr;
  {
    // first call on this device: look up the array's device address (the
    // host-side name of a __device__ variable is not a device pointer)
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
        cudaGetLastError();
        return CAS_ERR_CUDA;
      }
      g_noalloc_addr[dev] = static_cast<int64_t*>(p);
    }
    partial = g_noalloc_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // an error the caller has not read yet stays theirs: report it, launch
  // nothing, and leave it pending for the caller's own check
  if (cudaPeekAtLastError() != cudaSuccess) return CAS_ERR_CUDA;
  cas::k_scan_partials<<<(unsigned)nparts, cas::kScanBlock, 0, s>>>(d_in, n - 1, partial);
  cas::k_scan_top<<<1, cas::kScanBlock, 0, s>>>(partial, nparts, nullptr);
  cas::k_scan_apply<<<(unsigned)nparts, cas::kScanBlock, 0, s>>>(d_in, n - 1, partial, d_out, n);
  // a launch error here is this call's own: read it, and report it by status
  return cudaGetLastError() == cudaSuccess ? CAS_OK : CAS_ERR_CUDA;
}
