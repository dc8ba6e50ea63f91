// Sorting networks for the small buckets of the bucketed ESC kernel.
//
// A lane sorts one bucket of at most 8 (column, value) pairs.  Each pair is
// packed into one 32-bit word: the column's offset inside its bucket (below
// 2^23, since a bucket spans a 32-bit column range shifted down by at least 9
// bits) shifted up by 3, and the pair's slot 0..7 in the low 3 bits.  Words
// of distinct columns order as the columns do, and words of one column order
// by slot, so a network on the words is a stable sort of the pairs, and a
// comparator is one min and one max.  Empty inputs are 0xFFFFFFFF, which
// sorts last.
//
// The networks: Batcher's odd-even merge sort for 8 inputs (19 comparators)
// and optimal networks for 4 (5 comparators) and 6 inputs (12 comparators).
// This header is plain C++ outside nvcc, so the CPU tests check each network
// on every 0/1 input (the 0-1 principle) and on random words.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#define CAS_HD inline
#else
#define CAS_HD __host__ __device__ __forceinline__
#endif

namespace cas {

CAS_HD uint32_t sortnet_pack(uint32_t offset, int slot) { return (offset << 3) | (uint32_t)slot; }
CAS_HD uint32_t sortnet_offset(uint32_t w) { return w >> 3; }
CAS_HD int sortnet_slot(uint32_t w) { return (int)(w & 7u); }

CAS_HD void cmpx(uint32_t& a, uint32_t& b) {
  const uint32_t lo = a < b ? a : b;
  b = a < b ? b : a;
  a = lo;
}

CAS_HD void sort_net(uint32_t (&w)[4]) {
  cmpx(w[0], w[1]); cmpx(w[2], w[3]);
  cmpx(w[0], w[2]); cmpx(w[1], w[3]);
  cmpx(w[1], w[2]);
}

CAS_HD void sort_net(uint32_t (&w)[6]) {
  cmpx(w[0], w[5]); cmpx(w[1], w[3]); cmpx(w[2], w[4]);
  cmpx(w[1], w[2]); cmpx(w[3], w[4]);
  cmpx(w[0], w[3]); cmpx(w[2], w[5]);
  cmpx(w[0], w[1]); cmpx(w[2], w[3]); cmpx(w[4], w[5]);
  cmpx(w[1], w[2]); cmpx(w[3], w[4]);
}

CAS_HD void sort_net(uint32_t (&w)[8]) {
  cmpx(w[0], w[1]); cmpx(w[2], w[3]); cmpx(w[4], w[5]); cmpx(w[6], w[7]);
  cmpx(w[0], w[2]); cmpx(w[1], w[3]); cmpx(w[4], w[6]); cmpx(w[5], w[7]);
  cmpx(w[1], w[2]); cmpx(w[5], w[6]);
  cmpx(w[0], w[4]); cmpx(w[1], w[5]); cmpx(w[2], w[6]); cmpx(w[3], w[7]);
  cmpx(w[2], w[4]); cmpx(w[3], w[5]);
  cmpx(w[1], w[2]); cmpx(w[3], w[4]); cmpx(w[5], w[6]);
}

}  // namespace cas

#undef CAS_HD
