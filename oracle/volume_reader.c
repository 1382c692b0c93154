/*
 * Readers of the filter's output files for the render oracle — TEST
 * INFRASTRUCTURE ONLY (see oracle.h).
 *
 * NanoVDB: an uncompressed file as io::writeGrid lays it out (16-byte header,
 * 176-byte grid metadata, grid name, grid buffer), with voxel lookups that
 * walk the tree from the root tile table through the upper (32^3) and lower
 * (16^3) internal nodes to the 8^3 leaf, following NanoVDB's published node
 * layout (version 32.3) and ReadAccessor::getValue semantics: a missing child
 * yields the tile value stored in its parent's table.  The library under test
 * reads leaves through a flat block index instead, so the two lookups are
 * independent.
 *
 * Brick grid: the reference's ".brickgrid" file, a cereal 1.3.2
 * PortableBinary archive of CHostBrickGrid (serialization.cpp:37-40): one
 * byte 1 (little-endian payload), the mat4 transform (16 floats), n_bricks
 * (3 uint32), min_maj (2 floats), brick_counter (uint64), then indirection,
 * range (uint32) and atlas (uint8), each a Buf3D (stride as 3 uint32, then a
 * std::vector: uint64 element count and the elements), and range_mipmaps (a
 * uint64 count of uint32 Buf3Ds).  orc_build_bricks restates the
 * construction (host_grid_brick.cpp:61-152, common.hpp:23-53) one brick
 * after the other.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

#define NVDB_MAGIC 0x304244566f6e614eull
#define GRID_SIZE 672u
#define TREE_SIZE 64u
#define ROOT_SIZE 160u
#define TILE_SIZE 64u
#define UPPER_HDR 8320u
#define LOWER_HDR 1152u
#define LEAF_SIZE 16544u

static uint64_t rd64(const uint8_t* p) { uint64_t v; memcpy(&v, p, 8); return v; }
static uint32_t rd32(const uint8_t* p) { uint32_t v; memcpy(&v, p, 4); return v; }
static int32_t rdi32(const uint8_t* p) { int32_t v; memcpy(&v, p, 4); return v; }

int oi_nvdb_read(const char* path, oi_nvdb* g) {
  memset(g, 0, sizeof(*g));
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  uint8_t hdr[16], meta[176];
  if (fread(hdr, 1, 16, f) != 16 || fread(meta, 1, 176, f) != 176 || rd64(hdr) != NVDB_MAGIC) { fclose(f); return -2; }
  uint16_t codec;
  memcpy(&codec, hdr + 14, 2);
  uint64_t gridSize = rd64(meta);
  uint32_t nameSize = rd32(meta + 136);
  if (codec != 0 || gridSize < GRID_SIZE + TREE_SIZE + ROOT_SIZE || gridSize > (1ull << 40) || nameSize > (1u << 20)) {
    fclose(f);
    return -3;
  }
  if (fseek(f, (long)nameSize, SEEK_CUR) != 0) { fclose(f); return -4; }
  g->buf = (uint8_t*)malloc(gridSize);
  if (!g->buf || fread(g->buf, 1, gridSize, f) != gridSize) { fclose(f); free(g->buf); g->buf = NULL; return -5; }
  fclose(f);
  g->size = gridSize;
  const uint8_t* G = g->buf;
  if (rd64(G) != NVDB_MAGIC || rd64(G + 32) != gridSize || rd32(G + 636) != 18u /* Vec4d */) {
    oi_nvdb_free(g);
    return -6;
  }
  memcpy(g->matF, G + 296, 36);
  memcpy(g->vecF, G + 368, 12);
  memcpy(g->worldBBox, G + 560, 48);
  const uint8_t* T = G + GRID_SIZE;
  g->leafOff = GRID_SIZE + rd64(T);
  g->rootOff = GRID_SIZE + rd64(T + 24);
  g->leafCount = rd32(T + 32);
  g->voxelCount = rd64(T + 56);
  if (g->rootOff + ROOT_SIZE > gridSize || g->leafOff + (uint64_t)g->leafCount * LEAF_SIZE > gridSize) {
    oi_nvdb_free(g);
    return -7;
  }
  const uint8_t* R = G + g->rootOff;
  for (int k = 0; k < 6; ++k) g->indexBBox[k] = rdi32(R + 4 * k);
  g->tableSize = rd32(R + 24);
  if (g->rootOff + ROOT_SIZE + (uint64_t)g->tableSize * TILE_SIZE > gridSize) { oi_nvdb_free(g); return -8; }
  memcpy(g->background, R + 32, 32);
  return 0;
}

void oi_nvdb_free(oi_nvdb* g) {
  free(g->buf);
  memset(g, 0, sizeof(*g));
}

static int bit(const uint8_t* words, uint32_t i) { return (int)((rd64(words + 8 * (i >> 6)) >> (i & 63)) & 1u); }

void oi_nvdb_value(const oi_nvdb* g, int x, int y, int z, uint8_t out[32]) {
  const uint8_t* R = g->buf + g->rootOff;
  const uint64_t key = ((uint64_t)((uint32_t)z >> 12)) | ((uint64_t)((uint32_t)y >> 12) << 21) |
                       ((uint64_t)((uint32_t)x >> 12) << 42);
  memcpy(out, g->background, 32);
  for (uint32_t i = 0; i < g->tableSize; ++i) {
    const uint8_t* tile = R + ROOT_SIZE + (size_t)i * TILE_SIZE;
    if (rd64(tile) != key) continue;
    int64_t child;
    memcpy(&child, tile + 8, 8);
    if (child == 0) { memcpy(out, tile + 24, 32); return; }
    const uint8_t* U = R + child;
    const uint32_t ui = (((uint32_t)x & 4095u) >> 7) << 10 | (((uint32_t)y & 4095u) >> 7) << 5 | (((uint32_t)z & 4095u) >> 7);
    const uint8_t* ue = U + UPPER_HDR + 32u * ui;
    if (!bit(U + 32 + 4096, ui)) { memcpy(out, ue, 32); return; }
    int64_t off;
    memcpy(&off, ue, 8);
    const uint8_t* Lw = U + off;
    const uint32_t li = (((uint32_t)x & 127u) >> 3) << 8 | (((uint32_t)y & 127u) >> 3) << 4 | (((uint32_t)z & 127u) >> 3);
    const uint8_t* le = Lw + LOWER_HDR + 32u * li;
    if (!bit(Lw + 32 + 512, li)) { memcpy(out, le, 32); return; }
    memcpy(&off, le, 8);
    const uint8_t* Lf = Lw + off;
    const uint32_t vi = ((uint32_t)x & 7u) << 6 | ((uint32_t)y & 7u) << 3 | ((uint32_t)z & 7u);
    memcpy(out, Lf + 160 + 32u * vi, 32);
    return;
  }
}

float oi_nvdb_max_density(const oi_nvdb* g) {
  float m = 0.0f;
  for (uint32_t l = 0; l < g->leafCount; ++l) {
    const uint8_t* lf = g->buf + g->leafOff + (size_t)l * LEAF_SIZE + 160;
    for (int i = 0; i < 512; ++i) {
      float d;
      memcpy(&d, lf + 32 * i, 4);
      m = fmaxf(d, m);
    }
  }
  return m;
}

/* One Buf3D: its stride and a vector of `esize`-byte elements, whose count
 * must equal the stride's product; *out receives a malloc'd copy. */
static int read_buf3d(FILE* f, uint32_t stride[3], size_t esize, void** out) {
  uint64_t n = 0;
  if (fread(stride, 4, 3, f) != 3 || fread(&n, 8, 1, f) != 1) return 0;
  if (n != (uint64_t)stride[0] * stride[1] * stride[2] || n > ((uint64_t)1 << 34)) return 0;
  *out = malloc(n ? n * esize : 1);
  return *out && fread(*out, esize, n, f) == n;
}

int oi_bricks_read(const char* path, oi_bricks* b) {
  memset(b, 0, sizeof(*b));
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  uint8_t little = 0;
  float transform[16];
  uint64_t count = 0;
  uint32_t st[3];
  int ok = fread(&little, 1, 1, f) == 1 && little == 1 && fread(transform, 4, 16, f) == 16;
  ok = ok && fread(b->nb, 4, 3, f) == 3 && fread(&b->minorant, 4, 1, f) == 1 && fread(&b->majorant, 4, 1, f) == 1;
  ok = ok && fread(&count, 8, 1, f) == 1;
  for (int k = 0; ok && k < 3; ++k) ok = b->nb[k] > 0 && b->nb[k] < 1024 && (b->nb[k] & 7u) == 0;
  b->count = (uint32_t)count;
  ok = ok && read_buf3d(f, st, 4, (void**)&b->ind) && st[0] == b->nb[0] && st[1] == b->nb[1] && st[2] == b->nb[2];
  ok = ok && read_buf3d(f, st, 4, (void**)&b->range) && st[0] == b->nb[0] && st[1] == b->nb[1] && st[2] == b->nb[2];
  ok = ok && read_buf3d(f, b->ad, 1, (void**)&b->atlas);
  uint64_t nm = 0;
  ok = ok && fread(&nm, 8, 1, f) == 1 && nm == 3;
  for (int i = 0; ok && i < 3; ++i)
    ok = read_buf3d(f, st, 4, (void**)&b->mips[i]) && st[0] == b->nb[0] >> (i + 1) && st[1] == b->nb[1] >> (i + 1) &&
         st[2] == b->nb[2] >> (i + 1);
  fclose(f);
  if (!ok) {
    oi_bricks_free(b);
    return -2;
  }
  return 0;
}

void oi_bricks_free(oi_bricks* b) {
  free(b->ind);
  free(b->range);
  for (int i = 0; i < 3; ++i) free(b->mips[i]);
  free(b->atlas);
  memset(b, 0, sizeof(*b));
}
