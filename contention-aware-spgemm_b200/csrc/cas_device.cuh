// Device-side building blocks shared by the casgemm kernels (sm_100a).
//
//  * value traits for the two arithmetic modes: fp64 in / fp64 out (the
//    reference's my_rat_t, src/inc/store.h:20) and int32 in / int64 out;
//  * warp and block scans / reductions;
//  * warp-aggregated atomic counters (one atomic per distinct target per warp);
//  * a block-wide stable LSD radix sort of 64-bit items whose upper 32 bits are
//    the column key and lower 32 bits a payload index — the GPU form of the
//    reference's radix_sort_keyval_toggling_unrolling
//    (src/mm/mm_utils.c:1273-1375): 8-bit digits, only as many passes as the
//    key range needs, early-out when every key is equal.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cas {

constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;

// Error codes written by device-side guards (never a trap: the kernel skips
// the offending work and the host turns the code into a status).
enum DevErr : int32_t {
  kDevOk = 0,
  kDevRowOverflow = 1,   // a row produced more entries than its symbolic count
  kDevRowUnderflow = 2,  // a row produced fewer entries than its symbolic count
  kDevCapacity = 3,      // a row reached a kernel whose shared-memory capacity it exceeds
  kDevTableFull = 4,     // hash probing did not find a free slot
  kDevBadIndex = 5,      // a column index outside [0, num_col)
  kDevTimeout = 6,       // a bounded wait on another block gave up
};

struct DevStatus {
  int32_t err;
  int32_t kernel;
  int64_t row;
};

__device__ __forceinline__ void dev_report(DevStatus* st, int32_t code, int32_t kernel, int64_t row) {
  if (atomicCAS(&st->err, 0, code) == 0) {
    st->kernel = kernel;
    st->row = row;
  }
}

// ----------------------------------------------------------- value traits
template <typename VIn>
struct Acc;
template <>
struct Acc<double> {
  using T = double;
  __device__ __forceinline__ static T mul(double a, double b) { return a * b; }
  __device__ __forceinline__ static void atomic_add(T* p, T v) { atomicAdd(p, v); }
};
template <>
struct Acc<int32_t> {
  using T = long long;
  __device__ __forceinline__ static T mul(int32_t a, int32_t b) { return (long long)a * (long long)b; }
  __device__ __forceinline__ static void atomic_add(T* p, T v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
  }
};

// Multiplicative hash into a table of 2^tbits slots (Knuth's golden-ratio
// constant; the high bits of the product are the best mixed).
__device__ __forceinline__ uint32_t hash_slot(uint32_t key, int tbits) {
  return (key * 0x9E3779B1u) >> (32 - tbits);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ------------------------------------------------------------ warp scans
template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T u = __shfl_up_sync(kFull, v, d);
    if (lane >= d) v += u;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
  return v;
}

__device__ __forceinline__ uint32_t warp_min_u32(uint32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_xor_sync(kFull, v, d));
  return v;
}
__device__ __forceinline__ uint32_t warp_max_u32(uint32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(kFull, v, d));
  return v;
}

// ----------------------------------------------------------- block scans
// Exclusive prefix sum over the block; `tmp` holds BLOCK/32 + 1 entries.
// Returns the exclusive prefix of this thread, writes the block total.
template <int BLOCK, typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* tmp, T& total) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = warp_inclusive_sum(v);
  if (lane == 31) tmp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < NW ? tmp[lane] : T(0);
    T wi = warp_inclusive_sum(w);
    if (lane < NW) tmp[lane] = wi - w;
    if (lane == NW - 1) tmp[NW] = wi;
  }
  __syncthreads();
  T res = tmp[warp] + inc - v;
  total = tmp[NW];
  __syncthreads();
  return res;
}

template <int BLOCK, typename T>
__device__ __forceinline__ T block_sum(T v, T* tmp) {
  T total;
  block_exclusive_sum<BLOCK, T>(v, tmp, total);
  return total;
}

// -------------------------------------------- warp-aggregated atomic add
// All active lanes with the same `slot` are served by one atomicAdd issued by
// their lowest lane; returns the old value plus the lane's rank among its
// peers.  Used for bin cursors, where many lanes hit few counters.
__device__ __forceinline__ unsigned long long warp_aggregated_add(unsigned long long* base, int slot) {
  const unsigned active = __activemask();
  const unsigned peers = __match_any_sync(active, slot);
  const int leader = __ffs(peers) - 1;
  const int lane = threadIdx.x & 31;
  unsigned long long old = 0;
  if (lane == leader) old = atomicAdd(base + slot, (unsigned long long)__popc(peers));
  old = __shfl_sync(peers, old, leader);
  return old + __popc(peers & lanemask_lt());
}

// ------------------------------------------------------ block radix sort
// Stable LSD radix sort of n items (n <= 65535 per warp segment) in shared
// memory.  item = (key << 32) | payload; digits are taken from
// (key - kmin), passes = ceil(bits(kmax - kmin) / 8).  `a` holds the input;
// `b` is scratch of the same length; hist holds (BLOCK/32)*256 uint16 counters.
// Returns the buffer that holds the sorted items.
//
// Each warp owns a contiguous segment of the items and processes it 32 at a
// time, so (warp, round, lane) is the input order; a digit's output slot is
// (all smaller digits) + (same digit in earlier warps) + (same digit earlier in
// this warp), which keeps the sort stable.  Lanes with the same digit in a
// round find each other with __match_any_sync.
template <int BLOCK>
__device__ uint64_t* block_radix_sort(uint64_t* a, uint64_t* b, int n, uint32_t kmin, uint32_t kmax,
                                      uint16_t* hist, int* tmp) {
  constexpr int NW = BLOCK / 32;
  static_assert(BLOCK >= 256, "digit scan uses one thread per digit");
  if (n < 2 || kmax == kmin) return a;  // all keys equal: already sorted
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t range = kmax - kmin;
  const int bits = 32 - __clz(range);
  const int passes = (bits + 7) >> 3;
  const int seg = ((n + NW - 1) / NW + 31) & ~31;
  const int s0 = min(n, warp * seg), s1 = min(n, s0 + seg);
  uint64_t* in = a;
  uint64_t* out = b;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    for (int i = threadIdx.x; i < NW * 256; i += BLOCK) hist[i] = 0;
    __syncthreads();
    uint16_t* h = hist + warp * 256;
    for (int base = s0; base < s1; base += 32) {
      const int i = base + lane;
      const bool valid = i < s1;
      const int d = valid ? (int)((((uint32_t)(in[i] >> 32) - kmin) >> shift) & 0xFF) : 256 + lane;
      const unsigned peers = __match_any_sync(kFull, d);
      if (valid && lane == __ffs(peers) - 1) h[d] = (uint16_t)(h[d] + __popc(peers));
      __syncwarp();
    }
    __syncthreads();
    // digit-major, warp-minor exclusive offsets
    int tot = 0;
    if (threadIdx.x < 256) {
      for (int w = 0; w < NW; ++w) tot += hist[w * 256 + threadIdx.x];
    }
    int total;
    const int dbase = block_exclusive_sum<BLOCK, int>(threadIdx.x < 256 ? tot : 0, tmp, total);
    if (threadIdx.x < 256) {
      int run = dbase;
      for (int w = 0; w < NW; ++w) {
        const int c = hist[w * 256 + threadIdx.x];
        hist[w * 256 + threadIdx.x] = (uint16_t)run;
        run += c;
      }
    }
    __syncthreads();
    // NOTE: offsets are < n <= 65535, so uint16 holds them.
    for (int base = s0; base < s1; base += 32) {
      const int i = base + lane;
      const bool valid = i < s1;
      const uint64_t it = valid ? in[i] : 0;
      const int d = valid ? (int)((((uint32_t)(it >> 32) - kmin) >> shift) & 0xFF) : 256 + lane;
      const unsigned peers = __match_any_sync(kFull, d);
      int pos = 0;
      if (valid) pos = h[d] + __popc(peers & lanemask_lt());
      __syncwarp();
      if (valid) {
        out[pos] = it;
        if (lane == __ffs(peers) - 1) h[d] = (uint16_t)(h[d] + __popc(peers));
      }
      __syncwarp();
    }
    __syncthreads();
    uint64_t* t = in;
    in = out;
    out = t;
  }
  return in;
}

// Lower bound of `v` in the sorted int32 range [lo, hi) of global memory.
__device__ __forceinline__ int64_t lower_bound_g(const int32_t* __restrict__ a, int64_t lo, int64_t hi, int32_t v) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

}  // namespace cas
