// Stable LSD radix sort of (uint64 key, uint32 value) pairs on the device.
// See radix_sort.cu.
#pragma once
#include "runtime.h"

namespace r2 {

// Device scratch of the sort, grown on demand and kept between sorts.
struct RadixSortScratch {
  DBuf<uint64_t> keysAlt;
  DBuf<uint32_t> valsAlt;
  DBuf<uint32_t> hist;      // digit-major block histograms, then their exclusive prefix
  DBuf<uint32_t> partials;  // per-partition sums of the prefix pass
  void reserve(uint32_t n);
};

// data[0..n) becomes its exclusive prefix sum (n <= 2^24; partials: scratch,
// grown as needed), with the sort's reduce-then-scan kernels.
void exclusive_scan_inplace(uint32_t* data, uint32_t n, DBuf<uint32_t>* partials, cudaStream_t s);

// Sorts n pairs ascending by the low `bits` bits of the keys (1..64), stably:
// equal keys keep their input order.  In place: keys/vals hold the sorted
// pairs when the stream reaches the end of the sort.  Returns the number of
// kernels launched.
int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint32_t n, int bits, RadixSortScratch* scratch,
                      cudaStream_t s);

}  // namespace r2
