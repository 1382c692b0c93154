// Filter output stage on the device: active topology, NanoVDB leaf gather and
// the brick grid (see volume.h).
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>


#include "filter_math.h"
#include "radix_sort.cuh"
#include "volume.h"

namespace r2 {
namespace {

__device__ __forceinline__ bool is_corner(int x, int y, int z, int nx, int ny, int nz) {
  return (x == 0 || x == nx - 1) && (y == 0 || y == ny - 1) && (z == 0 || z == nz - 1);
}

// Density as stored in the grid: active voxels keep theirs, everything else
// (inactive or outside the index box) reads the background density 0.
__device__ __forceinline__ float grid_density(const r2_voxel* d, int x, int y, int z, int nx, int ny, int nz) {
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0.0f;
  float v = __ldg(&d[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny].density);
  return (v > 0.0f || is_corner(x, y, z, nx, ny, nz)) ? v : 0.0f;
}

__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// One warp per 8^3 block: lane l covers x offset l>>2 and the 16 (y, z)
// offsets (l&3)*16 .. +15, i.e. bits (l&3)*16.. of mask word x (NanoVDB voxel
// index (x<<6)|(y<<3)|z).  Active blocks are appended to `list`.
__global__ void __launch_bounds__(256) k_leaf_topology(const r2_voxel* __restrict__ d, int nx, int ny, int nz,
                                                       int Lx, int Ly, int Lz, uint64_t* __restrict__ masks,
                                                       uint32_t* __restrict__ list, uint32_t* __restrict__ counters) {
  const int lane = threadIdx.x & 31;
  const uint32_t nLeaves = (uint32_t)Lx * Ly * Lz;
  const uint32_t warpsTotal = gridDim.x * (blockDim.x >> 5);
  float lmin = INFINITY, lmax = -INFINITY;
  for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nLeaves; w += warpsTotal) {
    const int lx = (int)(w % (uint32_t)Lx), ly = (int)((w / (uint32_t)Lx) % (uint32_t)Ly), lz = (int)(w / ((uint32_t)Lx * Ly));
    const int ox = lx * 8, oy = ly * 8, oz = lz * 8;
    const int xo = lane >> 2;
    uint32_t bits = 0;
    for (int k = 0; k < 16; ++k) {
      const int yz = (lane & 3) * 16 + k;
      const int x = ox + xo, y = oy + (yz >> 3), z = oz + (yz & 7);
      if (x < nx && y < ny && z < nz) {
        const float v = __ldg(&d[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny].density);
        const bool act = v > 0.0f || is_corner(x, y, z, nx, ny, nz);
        bits |= (act ? 1u : 0u) << k;
        const float gv = act ? v : 0.0f;
        lmin = fminf(lmin, gv);
        lmax = fmaxf(lmax, gv);
      }
    }
    // assemble the 64-bit word of x offset xo from its four lanes
    const uint32_t b0 = __shfl_sync(0xFFFFFFFFu, bits, (lane & ~3) + 0);
    const uint32_t b1 = __shfl_sync(0xFFFFFFFFu, bits, (lane & ~3) + 1);
    const uint32_t b2 = __shfl_sync(0xFFFFFFFFu, bits, (lane & ~3) + 2);
    const uint32_t b3 = __shfl_sync(0xFFFFFFFFu, bits, (lane & ~3) + 3);
    const uint64_t word = (uint64_t)b0 | ((uint64_t)b1 << 16) | ((uint64_t)b2 << 32) | ((uint64_t)b3 << 48);
    if ((lane & 3) == 0) masks[(size_t)w * 8 + xo] = word;
    const bool any = __ballot_sync(0xFFFFFFFFu, bits != 0) != 0;
    if (any && lane == 0) list[atomicAdd(&counters[0], 1u)] = w;
  }
  // global minorant / majorant of the grid density
  for (int off = 16; off > 0; off >>= 1) {
    lmin = fminf(lmin, __shfl_xor_sync(0xFFFFFFFFu, lmin, off));
    lmax = fmaxf(lmax, __shfl_xor_sync(0xFFFFFFFFu, lmax, off));
  }
  if (lane == 0 && lmin <= lmax) {
    atomicMin(&counters[1], f2ord(lmin));
    atomicMax(&counters[2], f2ord(lmax));
  }
}

// One warp per active block: gathers its 512 payloads in NanoVDB order
// (inactive voxels = background).
__global__ void __launch_bounds__(256) k_leaf_gather(const r2_voxel* __restrict__ d, int nx, int ny, int nz, int Lx,
                                                     int Ly, const uint64_t* __restrict__ masks,
                                                     const uint32_t* __restrict__ list, uint32_t count,
                                                     r2_voxel* __restrict__ values) {
  const int lane = threadIdx.x & 31;
  const uint32_t warpsTotal = gridDim.x * (blockDim.x >> 5);
  const r2_voxel bg = empty_voxel();
  for (uint32_t s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < count; s += warpsTotal) {
    const uint32_t w = list[s];
    const int ox = (int)(w % (uint32_t)Lx) * 8, oy = (int)((w / (uint32_t)Lx) % (uint32_t)Ly) * 8,
              oz = (int)(w / ((uint32_t)Lx * Ly)) * 8;
    for (int i = lane; i < 512; i += 32) {
      const int x = ox + (i >> 6), y = oy + ((i >> 3) & 7), z = oz + (i & 7);
      const bool act = (masks[(size_t)w * 8 + (i >> 6)] >> (i & 63)) & 1ull;
      r2_voxel v = bg;
      if (act) v = d[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny];
      const uint4* src = reinterpret_cast<const uint4*>(&v);
      uint4* dst = reinterpret_cast<uint4*>(values + (size_t)s * 512 + i);
      dst[0] = src[0];
      dst[1] = src[1];
    }
  }
}

__device__ __forceinline__ uint32_t d_encode_range(float lo, float hi) {
  return (uint32_t)f32_to_f16_bits(lo) | ((uint32_t)f32_to_f16_bits(hi) << 16);
}

// Per brick: min/max over the dilated 10^3 neighbourhood (host_grid_brick.cpp:86-97).
__global__ void k_brick_range(const r2_voxel* __restrict__ d, int nx, int ny, int nz, uint32_t bx, uint32_t by,
                              uint32_t bz, uint32_t* __restrict__ range, uint32_t* __restrict__ nonconst) {
  const size_t nB = (size_t)bx * by * bz;
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < nB; b += (size_t)gridDim.x * blockDim.x) {
    const int x0 = (int)(b % bx) * 8, y0 = (int)((b / bx) % by) * 8, z0 = (int)(b / ((size_t)bx * by)) * 8;
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (int z = -1; z < 9; ++z)
      for (int y = -1; y < 9; ++y)
        for (int x = -1; x < 9; ++x) {
          const float v = grid_density(d, x0 + x, y0 + y, z0 + z, nx, ny, nz);
          lo = fminf(lo, v);
          hi = fmaxf(hi, v);
        }
    range[b] = d_encode_range(lo, hi);
    nonconst[b] = (hi == lo) ? 0u : 1u;
  }
}

__global__ void k_brick_atlas(const r2_voxel* __restrict__ d, int nx, int ny, int nz, uint32_t bx, uint32_t by,
                              uint32_t bz, const uint32_t* __restrict__ range, const uint32_t* __restrict__ nonconst,
                              const uint32_t* __restrict__ slot, uint32_t* __restrict__ indirection,
                              uint8_t* __restrict__ atlas, uint32_t ax, uint32_t ay) {
  const size_t nB = (size_t)bx * by * bz;
  // one block of 512 threads per brick
  for (size_t b = blockIdx.x; b < nB; b += gridDim.x) {
    if (!nonconst[b]) {
      if (threadIdx.x == 0) indirection[b] = 0;
      continue;
    }
    const uint32_t s = slot[b];
    const uint32_t px = s % bx, py = (s / bx) % by, pz = s / (bx * by);
    if (threadIdx.x == 0)
      indirection[b] = (min(px, kMaxBricks - 1) << (2 + 2 * kBrickBitsPerAxis)) |
                       (min(py, kMaxBricks - 1) << (2 + kBrickBitsPerAxis)) | (min(pz, kMaxBricks - 1) << 2);
    const float lo = f16_bits_to_f32((uint16_t)(range[b] & 0xFFFFu));
    const float hi = f16_bits_to_f32((uint16_t)(range[b] >> 16));
    const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;
    const int x0 = (int)(b % bx) * 8, y0 = (int)((b / bx) % by) * 8, z0 = (int)(b / ((size_t)bx * by)) * 8;
    const float v = grid_density(d, x0 + lx, y0 + ly, z0 + lz, nx, ny, nz);
    const float vn = fminf(fmaxf((v - lo) / (hi - lo), 0.0f), 1.0f);
    const uint8_t q = (uint8_t)roundf(255.0f * vn);
    const size_t ai = (size_t)(px * 8 + lx) + (size_t)(py * 8 + ly) * ax + (size_t)(pz * 8 + lz) * ax * ay;
    atlas[ai] = q;
  }
}

// Density min / max over the grid's voxels as the grid stores them
// (getMinorantMajorant, host_grid_brick.cpp:44-57): ordered words [0] min, [1] max.
__global__ void __launch_bounds__(256) k_density_minmax(const r2_voxel* __restrict__ d, int nx, int ny, int nz,
                                                        uint32_t* __restrict__ mm) {
  const size_t n = (size_t)nx * ny * nz;
  float lo = INFINITY, hi = -INFINITY;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % (size_t)nx), y = (int)((i / (size_t)nx) % (size_t)ny), z = (int)(i / ((size_t)nx * ny));
    const float v = grid_density(d, x, y, z, nx, ny, nz);
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, off));
    hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], f2ord(lo));
    atomicMax(&mm[1], f2ord(hi));
  }
}

__global__ void k_init_minmax(uint32_t* c) {
  c[0] = 0;
  c[1] = 0xFFFFFFFFu;
  c[2] = 0;
}

float ord2f(uint32_t o) {
  uint32_t b = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

}  // namespace

uint32_t encode_range(float lo, float hi) {
  return (uint32_t)f32_to_f16_bits(lo) | ((uint32_t)f32_to_f16_bits(hi) << 16);
}
void decode_range(uint32_t v, float* lo, float* hi) {
  *lo = f16_bits_to_f32((uint16_t)(v & 0xFFFFu));
  *hi = f16_bits_to_f32((uint16_t)(v >> 16));
}
uint32_t encode_ptr(uint32_t x, uint32_t y, uint32_t z) {
  auto c = [](uint32_t v) { return v < kMaxBricks ? v : kMaxBricks - 1; };
  return (c(x) << (2 + 2 * kBrickBitsPerAxis)) | (c(y) << (2 + kBrickBitsPerAxis)) | (c(z) << 2);
}
void decode_ptr(uint32_t v, uint32_t* x, uint32_t* y, uint32_t* z) {
  *x = (v >> (2 + 2 * kBrickBitsPerAxis)) & (kMaxBricks - 1);
  *y = (v >> (2 + kBrickBitsPerAxis)) & (kMaxBricks - 1);
  *z = (v >> 2) & (kMaxBricks - 1);
}

void extract_leaves(const r2_voxel* d_dense, const int32_t nv[3], cudaStream_t s, std::vector<nvdb::LeafBlock>* leaves,
                    std::vector<r2_voxel>* values) {
  const int Lx = (nv[0] + 7) / 8, Ly = (nv[1] + 7) / 8, Lz = (nv[2] + 7) / 8;
  const size_t nL = (size_t)Lx * Ly * Lz;
  DBuf<uint64_t> masks(nL * 8);
  DBuf<uint32_t> list(nL), counters(3);
  k_init_minmax<<<1, 1, 0, s>>>(counters.get());
  int blocks = (int)std::min<size_t>((nL + 7) / 8, (size_t)sm_count() * 16);
  k_leaf_topology<<<std::max(blocks, 1), 256, 0, s>>>(d_dense, nv[0], nv[1], nv[2], Lx, Ly, Lz, masks.get(),
                                                        list.get(), counters.get());
  uint32_t cnt[3];
  R2_CUDA(cudaMemcpyAsync(cnt, counters.get(), sizeof(cnt), cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaStreamSynchronize(s));
  const uint32_t count = cnt[0];
  DBuf<r2_voxel> vals((size_t)count * 512);
  if (count) {
    int gb = (int)std::min<size_t>((count + 7) / 8, (size_t)sm_count() * 16);
    k_leaf_gather<<<gb, 256, 0, s>>>(d_dense, nv[0], nv[1], nv[2], Lx, Ly, masks.get(), list.get(), count,
                                     vals.get());
  }
  std::vector<uint32_t> ids(count);
  std::vector<uint64_t> hmasks(nL * 8);
  if (count) list.download(ids.data(), count, s);
  masks.download(hmasks.data(), nL * 8, s);
  values->resize((size_t)count * 512);
  if (count) vals.download(values->data(), (size_t)count * 512, s);
  R2_CUDA(cudaStreamSynchronize(s));
  R2_CUDA(cudaGetLastError());
  leaves->resize(count);
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t w = ids[i];
    nvdb::LeafBlock& lb = (*leaves)[i];
    lb.origin[0] = (int32_t)(w % (uint32_t)Lx) * 8;
    lb.origin[1] = (int32_t)((w / (uint32_t)Lx) % (uint32_t)Ly) * 8;
    lb.origin[2] = (int32_t)(w / ((uint32_t)Lx * Ly)) * 8;
    memcpy(lb.mask, &hmasks[(size_t)w * 8], sizeof(lb.mask));
  }
}

void build_brick_grid(const r2_voxel* d_dense, const int32_t nv[3], cudaStream_t s, BrickGridHost* g) {
  uint32_t nb[3];
  for (int k = 0; k < 3; ++k) {
    uint32_t bricks = ((uint32_t)nv[k] + kBrickSize - 1) / kBrickSize;
    nb[k] = ((bricks + (1u << kNumMipmaps) - 1) >> kNumMipmaps) << kNumMipmaps;
    R2_REQUIRE(nb[k] < kMaxBricks, R2_ERR_UNSUPPORTED, "exceeded max brick count of 1024");
    g->nBricks[k] = nb[k];
  }
  const size_t nB = (size_t)nb[0] * nb[1] * nb[2];
  DBuf<uint32_t> range(nB), nonconst(nB), slot(nB), indirection(nB);
  int blocks = (int)std::min<size_t>((nB + 127) / 128, (size_t)sm_count() * 16);
  k_brick_range<<<std::max(blocks, 1), 128, 0, s>>>(d_dense, nv[0], nv[1], nv[2], nb[0], nb[1], nb[2], range.get(),
                                                    nonconst.get());
  R2_REQUIRE(nB <= (1u << 24), R2_ERR_UNSUPPORTED, "brick grid of more than 2^24 bricks");
  R2_CUDA(cudaMemcpyAsync(slot.get(), nonconst.get(), nB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  DBuf<uint32_t> partials;
  exclusive_scan_inplace(slot.get(), (uint32_t)nB, &partials, s);
  uint32_t lastSlot = 0, lastFlag = 0;
  R2_CUDA(cudaMemcpyAsync(&lastSlot, slot.get() + nB - 1, 4, cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaMemcpyAsync(&lastFlag, nonconst.get() + nB - 1, 4, cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaStreamSynchronize(s));
  g->brickCount = lastSlot + lastFlag;
  // atlas pruned in z to round(ceil(count / float(bx*by))) brick slices (host_grid_brick.cpp:126)
  const uint32_t zSlices = (uint32_t)roundf(ceilf((float)g->brickCount / (float)(nb[0] * nb[1])));
  g->atlasDim[0] = nb[0] * kBrickSize;
  g->atlasDim[1] = nb[1] * kBrickSize;
  g->atlasDim[2] = zSlices * kBrickSize;
  const size_t atlasN = (size_t)g->atlasDim[0] * g->atlasDim[1] * g->atlasDim[2];
  DBuf<uint8_t> atlas(std::max<size_t>(atlasN, 1));
  if (atlasN) R2_CUDA(cudaMemsetAsync(atlas.get(), 0, atlasN, s));
  int ab = (int)std::min<size_t>(nB, (size_t)sm_count() * 8);
  k_brick_atlas<<<std::max(ab, 1), 512, 0, s>>>(d_dense, nv[0], nv[1], nv[2], nb[0], nb[1], nb[2], range.get(),
                                                 nonconst.get(), slot.get(), indirection.get(), atlas.get(),
                                                 g->atlasDim[0], g->atlasDim[1]);
  DBuf<uint32_t> mm(2);
  const uint32_t mmInit[2] = {0xFFFFFFFFu, 0u};
  R2_CUDA(cudaMemcpyAsync(mm.get(), mmInit, sizeof(mmInit), cudaMemcpyHostToDevice, s));
  const size_t nvox = (size_t)nv[0] * nv[1] * nv[2];
  const int mb = (int)std::min<size_t>((nvox + 255) / 256, (size_t)sm_count() * 8);
  k_density_minmax<<<std::max(mb, 1), 256, 0, s>>>(d_dense, nv[0], nv[1], nv[2], mm.get());
  uint32_t mmHost[2];
  R2_CUDA(cudaMemcpyAsync(mmHost, mm.get(), sizeof(mmHost), cudaMemcpyDeviceToHost, s));
  g->range.resize(nB);
  g->indirection.resize(nB);
  g->atlas.resize(atlasN);
  range.download(g->range.data(), nB, s);
  indirection.download(g->indirection.data(), nB, s);
  if (atlasN) atlas.download(g->atlas.data(), atlasN, s);
  R2_CUDA(cudaStreamSynchronize(s));
  R2_CUDA(cudaGetLastError());
  // min/max mipmaps of the range texture (host_grid_brick.cpp:129-151)
  for (uint32_t i = 0; i < kNumMipmaps; ++i) {
    const uint32_t mx = nb[0] >> (i + 1), my = nb[1] >> (i + 1), mz = nb[2] >> (i + 1);
    const uint32_t sx = nb[0] >> i, sy = nb[1] >> i;
    const std::vector<uint32_t>& src = i == 0 ? g->range : g->mips[i - 1];
    std::vector<uint32_t>& dst = g->mips[i];
    dst.resize((size_t)mx * my * mz);
    for (uint32_t z = 0; z < mz; ++z)
      for (uint32_t y = 0; y < my; ++y)
        for (uint32_t x = 0; x < mx; ++x) {
          float lo = FLT_MAX, hi = -FLT_MAX;
          for (uint32_t dz = 0; dz < 2; ++dz)
            for (uint32_t dy = 0; dy < 2; ++dy)
              for (uint32_t dx = 0; dx < 2; ++dx) {
                float a, b;
                decode_range(src[(size_t)(2 * x + dx) + (size_t)(2 * y + dy) * sx + (size_t)(2 * z + dz) * sx * sy], &a,
                             &b);
                lo = std::min(lo, a);
                hi = std::max(hi, b);
              }
          dst[(size_t)x + (size_t)y * mx + (size_t)z * mx * my] = encode_range(lo, hi);
        }
  }
  g->minorant = ord2f(mmHost[0]);
  g->majorant = ord2f(mmHost[1]);
}

namespace {

struct Writer {
  FILE* f;
  bool ok = true;
  void bytes(const void* p, size_t n) { ok = ok && (n == 0 || fwrite(p, 1, n, f) == n); }
  template <typename T> void pod(const T& v) { bytes(&v, sizeof(T)); }
  template <typename T> void buf3d(const uint32_t stride[3], const std::vector<T>& data) {
    bytes(stride, 12);
    pod((uint64_t)data.size());
    bytes(data.data(), data.size() * sizeof(T));
  }
};

struct Reader {
  FILE* f;
  bool ok = true;
  void bytes(void* p, size_t n) { ok = ok && (n == 0 || fread(p, 1, n, f) == n); }
  template <typename T> void pod(T& v) { bytes(&v, sizeof(T)); }
  // A Buf3D whose element count must equal its stride's product and stay below `limit`.
  template <typename T> void buf3d(uint32_t stride[3], std::vector<T>& data, uint64_t limit) {
    uint64_t n = 0;
    bytes(stride, 12);
    pod(n);
    ok = ok && n == (uint64_t)stride[0] * stride[1] * stride[2] && n <= limit;
    if (!ok) return;
    data.resize(n);
    bytes(data.data(), n * sizeof(T));
  }
};

}  // namespace

void write_brick_grid(const std::string& path, const BrickGridHost& g) {
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path + " for writing");
  Writer w{f};
  w.pod((uint8_t)1);  // PortableBinaryOutputArchive: data stored little-endian
  w.bytes(g.transform, sizeof(g.transform));
  w.bytes(g.nBricks, 12);
  w.pod(g.minorant);
  w.pod(g.majorant);
  w.pod((uint64_t)g.brickCount);
  w.buf3d(g.nBricks, g.indirection);
  w.buf3d(g.nBricks, g.range);
  w.buf3d(g.atlasDim, g.atlas);
  w.pod((uint64_t)kNumMipmaps);
  for (uint32_t i = 0; i < kNumMipmaps; ++i) {
    const uint32_t ms[3] = {g.nBricks[0] >> (i + 1), g.nBricks[1] >> (i + 1), g.nBricks[2] >> (i + 1)};
    w.buf3d(ms, g.mips[i]);
  }
  const bool ok = (fclose(f) == 0) && w.ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

BrickGridHost read_brick_grid(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path);
  BrickGridHost g;
  Reader r{f};
  uint8_t little = 0;
  r.pod(little);
  r.ok = r.ok && little == 1;  // big-endian archives are not produced by the reference's x86 builds
  r.bytes(g.transform, sizeof(g.transform));
  r.bytes(g.nBricks, 12);
  r.pod(g.minorant);
  r.pod(g.majorant);
  uint64_t count = 0;
  r.pod(count);
  for (int k = 0; r.ok && k < 3; ++k) r.ok = g.nBricks[k] > 0 && g.nBricks[k] < kMaxBricks;
  const uint64_t nB = r.ok ? (uint64_t)g.nBricks[0] * g.nBricks[1] * g.nBricks[2] : 0;
  r.ok = r.ok && count <= nB;
  g.brickCount = (uint32_t)count;
  uint32_t st[3];
  r.buf3d(st, g.indirection, nB);
  r.ok = r.ok && st[0] == g.nBricks[0] && st[1] == g.nBricks[1] && st[2] == g.nBricks[2];
  r.buf3d(st, g.range, nB);
  r.ok = r.ok && st[0] == g.nBricks[0] && st[1] == g.nBricks[1] && st[2] == g.nBricks[2];
  r.buf3d(g.atlasDim, g.atlas, nB * kBrickSize * kBrickSize * kBrickSize);
  r.ok = r.ok && g.atlasDim[0] == g.nBricks[0] * kBrickSize && g.atlasDim[1] == g.nBricks[1] * kBrickSize &&
         g.atlasDim[2] % kBrickSize == 0 &&
         (uint64_t)(g.atlasDim[0] / kBrickSize) * (g.atlasDim[1] / kBrickSize) * (g.atlasDim[2] / kBrickSize) >= count;
  uint64_t nm = 0;
  r.pod(nm);
  r.ok = r.ok && nm == kNumMipmaps;
  for (uint32_t i = 0; r.ok && i < kNumMipmaps; ++i) {
    r.buf3d(st, g.mips[i], nB);
    r.ok = r.ok && st[0] == g.nBricks[0] >> (i + 1) && st[1] == g.nBricks[1] >> (i + 1) &&
           st[2] == g.nBricks[2] >> (i + 1);
  }
  fclose(f);
  R2_REQUIRE(r.ok, R2_ERR_IO, "corrupt or truncated brick grid " + path);
  return g;
}

std::string float_key(float v) {
  char b[64];
  snprintf(b, sizeof(b), "%f", (double)v);
  return b;
}

}  // namespace r2
