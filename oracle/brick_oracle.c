/*
 * Brick grid construction of the oracle — TEST INFRASTRUCTURE ONLY (see
 * oracle.h for who may call it).
 *
 * Restates CHostBrickGrid(const SOpenvdbData&, numVoxels)
 * (raytracer/src/grid_brick/host_grid_brick.cpp:61-152) with the encodings of
 * grid_brick/common.hpp:23-53, one brick after the other in z, y, x order.
 * The reference walks brick slices in parallel and hands out atlas slots with
 * an atomic counter, so its slot order varies from run to run; the sequential
 * order here is the one a single-threaded run of the reference produces, and
 * the one the library's exclusive scan produces.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "oracle_internal.h"

#define BRICK 8u
#define BITS 10u
#define MAXB (1u << BITS)

/* Density of the grid at (x, y, z): outside the index box the background 0. */
static float dens_at(const float* d, int nx, int ny, int nz, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0.0f;
  return d[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny];
}
static uint32_t enc_range(float lo, float hi) {
  return (uint32_t)oi_half_bits(lo) | ((uint32_t)oi_half_bits(hi) << 16);
}
static void dec_range(uint32_t v, float* lo, float* hi) {
  *lo = oi_half_to_float((uint16_t)(v & 0xFFFFu));
  *hi = oi_half_to_float((uint16_t)(v >> 16));
}
static uint32_t enc_ptr(uint32_t x, uint32_t y, uint32_t z) {
  x = x < MAXB ? x : MAXB - 1;
  y = y < MAXB ? y : MAXB - 1;
  z = z < MAXB ? z : MAXB - 1;
  return (x << (2 + 2 * BITS)) | (y << (2 + BITS)) | (z << 2);
}
/* encode_voxel: round(255 * clamp((v - lo) / (hi - lo), 0, 1)); a zero-width
 * decoded range (two densities that round to one half) maps v = lo to 0 and
 * v > lo to 255. */
static uint8_t enc_voxel(float v, float lo, float hi) {
  const float t = fminf(fmaxf((v - lo) / (hi - lo), 0.0f), 1.0f);
  return (uint8_t)roundf(255.0f * t);
}
static uint32_t div_up(uint32_t a, uint32_t b) { return (uint32_t)ceilf((float)a / (float)b); }

int orc_build_bricks(const float* dens, int nx, int ny, int nz, uint32_t* nb, uint32_t* ind, uint32_t* range,
                     uint32_t* mip0, uint32_t* mip1, uint32_t* mip2, uint8_t* atlas, uint32_t* ad,
                     uint64_t* count, float* minmaj) {
  const uint32_t nv[3] = {(uint32_t)nx, (uint32_t)ny, (uint32_t)nz};
  for (int k = 0; k < 3; ++k) {
    nb[k] = div_up(div_up(nv[k], BRICK), 8u) * 8u;
    if (nb[k] >= MAXB) return -1;
  }
  if (!ind) return 0;
  /* getMinorantMajorant: over the grid's voxels */
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (size_t i = 0; i < (size_t)nx * ny * nz; ++i) {
    mn = fminf(mn, dens[i]);
    mx = fmaxf(mx, dens[i]);
  }
  minmaj[0] = mn;
  minmaj[1] = mx;
  const size_t ax = (size_t)nb[0] * BRICK, ay = (size_t)nb[1] * BRICK;
  memset(atlas, 0, ax * ay * (size_t)nb[2] * BRICK);
  uint64_t counter = 0;
  for (uint32_t bz = 0; bz < nb[2]; ++bz)
    for (uint32_t by = 0; by < nb[1]; ++by)
      for (uint32_t bx = 0; bx < nb[0]; ++bx) {
        const size_t b = bx + (size_t)by * nb[0] + (size_t)bz * nb[0] * nb[1];
        ind[b] = 0;
        float lmin = FLT_MAX, lmax = -FLT_MAX;
        for (int z = -1; z < (int)BRICK + 1; ++z)
          for (int y = -1; y < (int)BRICK + 1; ++y)
            for (int x = -1; x < (int)BRICK + 1; ++x) {
              const float v = dens_at(dens, nx, ny, nz, (int)(bx * BRICK) + x, (int)(by * BRICK) + y,
                                      (int)(bz * BRICK) + z);
              lmin = fminf(lmin, v);
              lmax = fmaxf(lmax, v);
            }
        range[b] = enc_range(lmin, lmax);
        if (lmax == lmin) continue;
        const uint64_t id = counter++;
        const uint32_t px = (uint32_t)(id % nb[0]), py = (uint32_t)((id / nb[0]) % nb[1]),
                       pz = (uint32_t)(id / ((uint64_t)nb[0] * nb[1]));
        ind[b] = enc_ptr(px, py, pz);
        float lo, hi;
        dec_range(range[b], &lo, &hi);
        for (uint32_t z = 0; z < BRICK; ++z)
          for (uint32_t y = 0; y < BRICK; ++y)
            for (uint32_t x = 0; x < BRICK; ++x) {
              const float v = dens_at(dens, nx, ny, nz, (int)(bx * BRICK + x), (int)(by * BRICK + y),
                                      (int)(bz * BRICK + z));
              atlas[(px * BRICK + x) + (py * BRICK + y) * ax + (pz * BRICK + z) * ax * ay] = enc_voxel(v, lo, hi);
            }
      }
  *count = counter;
  ad[0] = (uint32_t)ax;
  ad[1] = (uint32_t)ay;
  ad[2] = BRICK * (uint32_t)roundf(ceilf((float)counter / (float)(nb[0] * nb[1])));
  uint32_t* mips[3] = {mip0, mip1, mip2};
  for (uint32_t i = 0; i < 3; ++i) {
    const uint32_t mx3[3] = {nb[0] >> (i + 1), nb[1] >> (i + 1), nb[2] >> (i + 1)};
    const uint32_t sx = nb[0] >> i, sy = nb[1] >> i;
    const uint32_t* src = i == 0 ? range : mips[i - 1];
    for (uint32_t z = 0; z < mx3[2]; ++z)
      for (uint32_t y = 0; y < mx3[1]; ++y)
        for (uint32_t x = 0; x < mx3[0]; ++x) {
          float lo = FLT_MAX, hi = -FLT_MAX;
          for (uint32_t dz = 0; dz < 2; ++dz)
            for (uint32_t dy = 0; dy < 2; ++dy)
              for (uint32_t dx = 0; dx < 2; ++dx) {
                float a, c;
                dec_range(src[(2 * x + dx) + (size_t)(2 * y + dy) * sx + (size_t)(2 * z + dz) * sx * sy], &a, &c);
                lo = fminf(lo, a);
                hi = fmaxf(hi, c);
              }
          mips[i][x + (size_t)y * mx3[0] + (size_t)z * mx3[0] * mx3[1]] = enc_range(lo, hi);
        }
  }
  return 0;
}
