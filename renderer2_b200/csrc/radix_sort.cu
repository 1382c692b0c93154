// Stable LSD radix sort of (uint64 key, uint32 value) pairs, 8 bits per pass.
//
// One pass over digit d = (key >> shift) & 255:
//  1. k_rs_hist: each block counts the digits of its tile (kRsTile pairs) into
//     hist[d * nblocks + block].  In this digit-major order the exclusive
//     prefix sum of the whole array is, for each (digit, block), the first
//     output position of that block's keys with that digit.
//  2. k_rs_reduce, k_rs_partials, k_rs_down: that exclusive prefix sum
//     (reduce-then-scan over partitions of kScanPart words).
//  3. k_rs_scatter: each warp ranks its contiguous 512 pairs in input order
//     (keys with equal digits found with __match_any_sync, running counts per
//     warp and digit in shared memory), the warps' counts are offset by the
//     counts of the warps before them, and every pair is written to
//     prefix + rank.  Ranks follow the input order, so the sort is stable.
#include <utility>

#include "radix_sort.cuh"

namespace r2 {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 16;                    // pairs per thread
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 pairs per block
constexpr int kRsWarpTile = 32 * kRsItems;      // 512 consecutive pairs per warp
constexpr int kRsBins = 256;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanPart = kScanThreads * kScanItems;  // 4096 words per partition
static_assert(kRsThreads == kRsBins, "one thread per digit in the per-block passes");

__global__ void __launch_bounds__(kRsThreads)
    k_rs_hist(const uint64_t* __restrict__ keys, uint32_t n, int shift, uint32_t nblocks, uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[kRsBins];
  sh[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
#pragma unroll 4
  for (int i = 0; i < kRsItems; ++i) {
    const uint64_t k = base + (uint64_t)i * kRsThreads + threadIdx.x;
    if (k < n) atomicAdd(&sh[(uint32_t)(keys[k] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = sh[threadIdx.x];
}

// Exclusive scan of one value per thread over the block; *total gets the sum.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warpSums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? warpSums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) warpSums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t before = warp ? warpSums[warp - 1] : 0u;
  *total = warpSums[kScanThreads / 32 - 1];
  __syncthreads();  // warpSums is rewritten by the next call
  return before + x - v;
}

// partials[p] = sum of hist over partition p.
__global__ void __launch_bounds__(kScanThreads)
    k_rs_reduce(const uint32_t* __restrict__ hist, uint32_t L, uint32_t* __restrict__ partials) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanPart;
  uint32_t s = 0;
#pragma unroll 4
  for (int i = 0; i < kScanItems; ++i) {
    const uint64_t k = base + (uint64_t)i * kScanThreads + threadIdx.x;
    if (k < L) s += hist[k];
  }
  uint32_t total;
  block_exclusive_scan(s, &total);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Exclusive prefix of the partition sums (at most kScanPart of them), one block.
__global__ void __launch_bounds__(kScanThreads) k_rs_partials(uint32_t* __restrict__ partials, uint32_t np) {
  uint32_t v[kScanItems];
  uint32_t s = 0;
  const uint32_t b = threadIdx.x * kScanItems;  // consecutive words per thread, in order
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (b + i < np) ? partials[b + i] : 0u;
    s += v[i];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (b + i < np) partials[b + i] = run;
    run += v[i];
  }
}

// hist becomes its exclusive prefix sum: partition offset + scan within the partition.
__global__ void __launch_bounds__(kScanThreads)
    k_rs_down(uint32_t* __restrict__ hist, uint32_t L, const uint32_t* __restrict__ partials) {
  const uint64_t b = (uint64_t)blockIdx.x * kScanPart + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (b + i < L) ? hist[b + i] : 0u;
    s += v[i];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total) + partials[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (b + i < L) hist[b + i] = run;
    run += v[i];
  }
}

__global__ void __launch_bounds__(kRsThreads)
    k_rs_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
                 uint32_t* __restrict__ vout, uint32_t n, int shift, uint32_t nblocks,
                 const uint32_t* __restrict__ prefix) {
  __shared__ uint32_t cnt[kRsWarps][kRsBins];
  __shared__ uint32_t first[kRsBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kRsWarps * kRsBins; i += kRsThreads) (&cnt[0][0])[i] = 0u;
  __syncthreads();
  const uint64_t wbase = (uint64_t)blockIdx.x * kRsTile + (uint64_t)warp * kRsWarpTile;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t rank[kRsItems];
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    const uint64_t k = wbase + (uint64_t)r * 32 + lane;
    const bool ok = k < n;
    // lanes past the end form their own group (digit 256) and count nowhere
    const uint32_t d = ok ? ((uint32_t)(kin[k] >> shift) & 0xFFu) : (uint32_t)kRsBins;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    const uint32_t before = ok ? cnt[warp][d] : 0u;
    __syncwarp();
    if (ok && (peers & lt) == 0u) cnt[warp][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt);
  }
  __syncthreads();
  {  // per digit: the warps' counts become offsets, and the block's first position
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const uint32_t c = cnt[w][d];
      cnt[w][d] = run;
      run += c;
    }
    first[d] = prefix[(size_t)d * nblocks + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    const uint64_t k = wbase + (uint64_t)r * 32 + lane;
    if (k < n) {
      const uint64_t key = kin[k];
      const uint32_t d = (uint32_t)(key >> shift) & 0xFFu;
      const uint32_t pos = first[d] + cnt[warp][d] + rank[r];
      kout[pos] = key;
      vout[pos] = vin[k];
    }
  }
}

uint32_t rs_blocks(uint32_t n) { return (n + kRsTile - 1) / kRsTile; }

}  // namespace

void RadixSortScratch::reserve(uint32_t n) {
  keysAlt.reserve(n);
  valsAlt.reserve(n);
  const size_t L = (size_t)rs_blocks(n) * kRsBins;
  hist.reserve(L);
  partials.reserve((L + kScanPart - 1) / kScanPart);
}

void exclusive_scan_inplace(uint32_t* data, uint32_t n, DBuf<uint32_t>* partials, cudaStream_t s) {
  if (n == 0) return;
  const uint32_t np = (n + kScanPart - 1) / kScanPart;
  R2_REQUIRE(np <= (uint32_t)kScanPart, R2_ERR_UNSUPPORTED, "prefix sum of more than 2^24 words");
  partials->reserve(np);
  k_rs_reduce<<<np, kScanThreads, 0, s>>>(data, n, partials->get());
  k_rs_partials<<<1, kScanThreads, 0, s>>>(partials->get(), np);
  k_rs_down<<<np, kScanThreads, 0, s>>>(data, n, partials->get());
  R2_CUDA(cudaGetLastError());
}

int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint32_t n, int bits, RadixSortScratch* scr, cudaStream_t s) {
  R2_REQUIRE(bits >= 1 && bits <= 64, R2_ERR_INVALID_ARGUMENT, "radix sort key bits must be in [1, 64]");
  if (n <= 1) return 0;
  const uint32_t nb = rs_blocks(n);
  const size_t L = (size_t)nb * kRsBins;
  const uint32_t np = (uint32_t)((L + kScanPart - 1) / kScanPart);
  R2_REQUIRE(np <= (uint32_t)kScanPart, R2_ERR_UNSUPPORTED, "radix sort of more than 2^28 pairs");
  scr->reserve(n);
  uint64_t* kin = keys;
  uint64_t* kout = scr->keysAlt.get();
  uint32_t* vin = vals;
  uint32_t* vout = scr->valsAlt.get();
  uint32_t* hist = scr->hist.get();
  uint32_t* partials = scr->partials.get();
  const int passes = (bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_rs_hist<<<nb, kRsThreads, 0, s>>>(kin, n, shift, nb, hist);
    k_rs_reduce<<<np, kScanThreads, 0, s>>>(hist, (uint32_t)L, partials);
    k_rs_partials<<<1, kScanThreads, 0, s>>>(partials, np);
    k_rs_down<<<np, kScanThreads, 0, s>>>(hist, (uint32_t)L, partials);
    k_rs_scatter<<<nb, kRsThreads, 0, s>>>(kin, vin, kout, vout, n, shift, nb, hist);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  R2_CUDA(cudaGetLastError());
  if (kin != keys) {
    R2_CUDA(cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    R2_CUDA(cudaMemcpyAsync(vals, vin, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  return 5 * passes;
}

}  // namespace r2
