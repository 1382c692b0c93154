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
 * Brick grid: the library's own ".brickgrid" format (magic "R2BRICK1", brick
 * counts, atlas size, brick count, minorant, majorant, then the indirection,
 * range, three mip and atlas arrays).
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

int oi_bricks_read(const char* path, oi_bricks* b) {
  memset(b, 0, sizeof(*b));
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  char magic[8];
  int ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "R2BRICK1", 8) == 0;
  ok = ok && fread(b->nb, 4, 3, f) == 3 && fread(b->ad, 4, 3, f) == 3 && fread(&b->count, 4, 1, f) == 1;
  ok = ok && fread(&b->minorant, 4, 1, f) == 1 && fread(&b->majorant, 4, 1, f) == 1;
  for (int k = 0; ok && k < 3; ++k) ok = b->nb[k] > 0 && b->nb[k] < 1024 && (b->nb[k] & 7u) == 0 && b->ad[k] <= 8192;
  if (ok) {
    const size_t nB = (size_t)b->nb[0] * b->nb[1] * b->nb[2];
    b->ind = (uint32_t*)malloc(4 * nB);
    b->range = (uint32_t*)malloc(4 * nB);
    ok = b->ind && b->range && fread(b->ind, 4, nB, f) == nB && fread(b->range, 4, nB, f) == nB;
    for (int i = 0; ok && i < 3; ++i) {
      const size_t m = (size_t)(b->nb[0] >> (i + 1)) * (b->nb[1] >> (i + 1)) * (b->nb[2] >> (i + 1));
      b->mips[i] = (uint32_t*)malloc(4 * (m ? m : 1));
      ok = b->mips[i] && fread(b->mips[i], 4, m, f) == m;
    }
    const size_t an = (size_t)b->ad[0] * b->ad[1] * b->ad[2];
    b->atlas = (uint8_t*)malloc(an ? an : 1);
    ok = ok && b->atlas && fread(b->atlas, 1, an, f) == an;
  }
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
